"""bench.py's reference arm on CPU: one JSON line in the contract's shape,
its config built by the same function as the GPU arm's line (so the two
lines describe the same workload), and an end-to-end figure that moves no
bytes between host and device."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line_on_a_small_cylinder():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--div", "8",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, cwd=ROOT,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    sys.path.insert(0, ROOT)
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    args = bench.parse(["--div", "8"])
    args.partition = False
    prob = bench.build_problem(args.workload, args.div)
    want = bench.arm_config(args, 1, prob.nelem, prob.npoin, prob.nelem * 8, bench.working_set(prob, args.precision))
    assert d["config"] == want, (d["config"], want)
    assert "fits the 126 MB L2" in d["config"]["l2"]
