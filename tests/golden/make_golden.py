"""Generate tests/golden/data1_transitions.npz from the reference's own
law-160 Gauss-point trace tests/sma_explicit/data1.dat.

Run once in a checkout that has the reference tree (argument: its path).

data1.dat holds rows (|e|, F) where |e| is the norm of the deviatoric
logarithmic strain and F = 2G(|e| - eL*xS) the loading function of law 160
(sld_stress_model_160.f90:513-537) for the uniaxial_test parameters
E=1000, nu=0.3, eL=0.1, AS 90/150, SA 70/30, alpha=0, C=0
(tests/uniaxial_test/sm154_d1C.sld.dat:21).  With alpha = 0 and C = 0 the
state (xS, F_AS, F_SA) of a row is (|e| - F/2G)/eL, F, F.  The trace
interleaves many Gauss points (about 128 rows per step), so for each row in
which the martensite fraction changed we search the 400 preceding rows for
the predecessor state from which one law update at the row's |e| gives the
row's F.  The fixture stores, for every such row: the new |e|, the
predecessor state and the expected F and xS; plus the envelope statistics of
the whole file.  tests/test_oracle_golden.py replays each transition through
the C oracle's full 3-D law (eigen-decomposition, logs, return map).
"""
import json
import os
import sys

import numpy as np

E, NU, EL = 1000.0, 0.3, 0.1
TWOG = E / (1.0 + NU)
AUX = np.sqrt(2.0 / 3.0)
RS_AS, RF_AS, RS_SA, RF_SA = 90 * AUX, 150 * AUX, 70 * AUX, 30 * AUX
G1 = TWOG * EL
WINDOW = 400


def law_1d(en, xS0, F0):
    """One update of law 160 reduced to alpha = 0, C = 0 (both loading
    functions equal); used only to locate predecessors in the trace."""
    FAS = TWOG * (en - EL * xS0)
    kAS = FAS > F0 and FAS - RS_AS > 0 and xS0 < 1
    kSA = FAS < F0 and FAS - RS_SA < 0 and xS0 > 0
    if not (kAS or kSA):
        return xS0, FAS
    HAS, HSA = float(kAS), float(kSA)
    xS, dAS, dSA, it = xS0, 0.0, 0.0, 0
    Fd = FAS - F0
    rAS = (FAS - RF_AS) * dAS + HAS * Fd * (1 - xS)
    rSA = (FAS - RF_SA) * dSA - HSA * Fd * xS
    res = rAS ** 2 + rSA ** 2
    while it < 65 and res > 1e-8:
        it += 1
        m11 = -G1 * dAS - (HAS * Fd + HAS * (1 - xS) * G1) + (FAS - RF_AS)
        m12 = -G1 * dAS - (HAS * Fd + HAS * (1 - xS) * G1)
        m21 = -G1 * dSA - (HSA * Fd - HSA * xS * G1)
        m22 = -G1 * dSA - (HSA * Fd - HSA * xS * G1) + (FAS - RF_SA)
        det = m11 * m22 - m12 * m21
        s1 = (m22 * rAS - m12 * rSA) / det
        s2 = (-m21 * rAS + m11 * rSA) / det
        dAS -= s1
        dSA -= s2
        xS = xS + dSA + dAS
        FAS = TWOG * (en - EL * xS)
        Fd = FAS - F0
        rAS = (FAS - RF_AS) * dAS + HAS * Fd * (1 - xS)
        rSA = (FAS - RF_SA) * dSA - HSA * Fd * xS
        res = np.sqrt(rAS ** 2 + rSA ** 2)
    if it >= 65:
        return xS0, F0
    return min(max(xS, 0.0), 1.0), FAS


def main(ref_root):
    path = os.path.join(ref_root, "tests", "sma_explicit", "data1.dat")
    d = np.loadtxt(path, delimiter=",")
    en, F = d[:, 0], d[:, 1]
    xs = (en - F / TWOG) / EL
    rows = []
    for j in range(1, len(d)):
        lo = max(0, j - 16)
        if np.min(np.abs(xs[lo:j] - xs[j])) <= 1e-12:
            continue  # no transformation at this row
        best, bi = np.inf, -1
        for i in range(max(0, j - WINDOW), j):
            x1, F1 = law_1d(en[j], xs[i], F[i])
            e = abs(TWOG * (en[j] - EL * x1) - F[j])
            if e < best:
                best, bi = e, i
        rows.append((j, bi, en[j], xs[bi], F[bi], F[j], xs[j], best))
    r = np.array(rows)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data1_transitions.npz")
    np.savez_compressed(out, row=r[:, 0].astype(np.int32), pred=r[:, 1].astype(np.int32),
                        en_new=r[:, 2], xS0=r[:, 3], F0=r[:, 4], F_new=r[:, 5], xS_new=r[:, 6],
                        search_err=r[:, 7],
                        props=np.array([E, NU, EL, 90, 150, 0, 0, 0, 700, 70, 30, 0, 0, 0, 0, 10, 10, 0.0]))
    env = dict(rows=int(len(d)), en_max=float(en.max()), F_max=float(F.max()),
               xS_min=float(xs.min()), xS_max=float(xs.max()),
               elastic_slope_2G=TWOG, Rf_AS=float(RF_AS), transitions=int(len(rows)),
               transitions_within_1e9=int(np.sum(r[:, 7] < 1e-9)))
    with open(os.path.join(os.path.dirname(out), "data1_envelope.json"), "w") as fh:
        json.dump(env, fh, indent=1)
    print(json.dumps(env, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
