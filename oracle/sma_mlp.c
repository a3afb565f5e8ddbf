/*
 * sma_mlp.c -- FP64 restatement of the learned constitutive surrogate's
 * network: the checker of the library's BF16 tensor-core training and
 * inference kernels.
 *
 * TEST INFRASTRUCTURE ONLY: called by tests/ (gradient and forward checks)
 * and nothing else; the product never links it.
 *
 * The reference has no surrogate.  Its adjacent hook is the ANN framework's
 * forward pass through an external libtorch wrapper
 * (src/alya-ann/mod_ann_framework.f90:421-446, eval_r1), which has no
 * backward pass; the network here restates the published algorithms it is
 * built from: a multilayer perceptron trained by backpropagation (Rumelhart,
 * Hinton & Williams, Nature 323, 1986) with the SiLU activation
 * x * sigmoid(x) (Elfwing, Uchibe & Doya, Neural Networks 107, 2018).
 *
 * Network: 14 -> 64 -> 64 -> 64 -> 64 -> 13, SiLU after each hidden layer,
 * linear output.  Inputs and outputs are normalised per feature,
 *   xh = (x - mu_x) / sd_x,   yh = (y - mu_y) / sd_y,
 * and the loss is the mean over samples and outputs of (yh_pred - yh)^2.
 * Parameters use the library's padded flat layout (padding holds zero):
 *   W1 [64][16], b1 [64], W2 [64][64], b2 [64], W3 [64][64], b3 [64],
 *   W4 [64][64], b4 [64], W5 [16][64], b5 [16]          (14,608 values)
 * with W[o][i] the weight from input i to output o.  stats holds
 * mu_x[14], sd_x[14], mu_y[13], sd_y[13].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NIN 14
#define NOUT 13
#define H 64
#define KIN 16     /* padded input width  */
#define KOUT 16    /* padded output width */

enum {
  OW1 = 0, OB1 = OW1 + H * KIN, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H * H,
  OW4 = OB3 + H, OB4 = OW4 + H * H, OW5 = OB4 + H, OB5 = OW5 + KOUT * H, NPARAM = OB5 + KOUT
};

int orc_mlp_nparam(void) { return NPARAM; }

static double sigm(double z) { return 1.0 / (1.0 + exp(-z)); }

/* one sample: pre-activations z[l][64] (l = 0..3) and activations a[l][64],
 * output yh[13] (normalised) */
static void forward1(const double* p, const double* stats, const double* x, double xh[KIN],
                     double z[4][H], double a[4][H], double yh[KOUT])
{
  const double *mu_x = stats, *sd_x = stats + NIN;
  for (int i = 0; i < KIN; ++i) xh[i] = (i < NIN) ? (x[i] - mu_x[i]) / sd_x[i] : 0.0;
  const int ow[4] = {OW1, OW2, OW3, OW4}, ob[4] = {OB1, OB2, OB3, OB4};
  for (int l = 0; l < 4; ++l) {
    const int nin = (l == 0) ? KIN : H;
    const double* in = (l == 0) ? xh : a[l - 1];
    for (int o = 0; o < H; ++o) {
      double s = p[ob[l] + o];
      for (int i = 0; i < nin; ++i) s += p[ow[l] + o * nin + i] * in[i];
      z[l][o] = s;
      a[l][o] = s * sigm(s);
    }
  }
  for (int o = 0; o < KOUT; ++o) {
    double s = p[OB5 + o];
    for (int i = 0; i < H; ++i) s += p[OW5 + o * H + i] * a[3][i];
    yh[o] = s;
  }
}

/* raw outputs y (n, 13) of raw inputs x (n, 14) */
void orc_mlp_forward(const double* params, const double* stats, int64_t n, const double* x, double* y)
{
  const double *mu_y = stats + 2 * NIN, *sd_y = stats + 2 * NIN + NOUT;
  for (int64_t s = 0; s < n; ++s) {
    double xh[KIN], z[4][H], a[4][H], yh[KOUT];
    forward1(params, stats, x + NIN * s, xh, z, a, yh);
    for (int o = 0; o < NOUT; ++o) y[NOUT * s + o] = yh[o] * sd_y[o] + mu_y[o];
  }
}

/* loss of the batch and, if grad is not NULL, its gradient with respect to
 * every parameter (padded layout; the padding's gradient is zero) */
double orc_mlp_loss_grad(const double* params, const double* stats, int64_t n, const double* x,
                         const double* y, double* grad)
{
  const double *mu_y = stats + 2 * NIN, *sd_y = stats + 2 * NIN + NOUT;
  if (grad) memset(grad, 0, sizeof(double) * NPARAM);
  const double scale = 1.0 / ((double)n * NOUT);
  double loss = 0.0;
  const int ow[4] = {OW1, OW2, OW3, OW4}, ob[4] = {OB1, OB2, OB3, OB4};
  for (int64_t s = 0; s < n; ++s) {
    double xh[KIN], z[4][H], a[4][H], yh[KOUT], d5[KOUT], d[H], dn[H];
    forward1(params, stats, x + NIN * s, xh, z, a, yh);
    for (int o = 0; o < KOUT; ++o) {
      const double t = (o < NOUT) ? (y[NOUT * s + o] - mu_y[o]) / sd_y[o] : 0.0;
      const double e = (o < NOUT) ? yh[o] - t : 0.0;
      loss += e * e;
      d5[o] = 2.0 * e * scale;
    }
    if (!grad) continue;
    /* output layer */
    for (int o = 0; o < KOUT; ++o) {
      grad[OB5 + o] += d5[o];
      for (int i = 0; i < H; ++i) grad[OW5 + o * H + i] += d5[o] * a[3][i];
    }
    for (int i = 0; i < H; ++i) {
      double s = 0.0;
      for (int o = 0; o < KOUT; ++o) s += d5[o] * params[OW5 + o * H + i];
      const double sg = sigm(z[3][i]);
      d[i] = s * (sg * (1.0 + z[3][i] * (1.0 - sg)));          /* SiLU'(z) */
    }
    /* hidden layers 4..1 */
    for (int l = 3; l >= 0; --l) {
      const int nin = (l == 0) ? KIN : H;
      const double* in = (l == 0) ? xh : a[l - 1];
      for (int o = 0; o < H; ++o) {
        grad[ob[l] + o] += d[o];
        for (int i = 0; i < nin; ++i) grad[ow[l] + o * nin + i] += d[o] * in[i];
      }
      if (l == 0) break;
      for (int i = 0; i < H; ++i) {
        double t = 0.0;
        for (int o = 0; o < H; ++o) t += d[o] * params[ow[l] + o * H + i];
        const double sg = sigm(z[l - 1][i]);
        dn[i] = t * (sg * (1.0 + z[l - 1][i] * (1.0 - sg)));
      }
      memcpy(d, dn, sizeof d);
    }
  }
  return loss * scale;
}
