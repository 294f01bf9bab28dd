/* CPU restatement of the learned closure's arithmetic: the pointwise MLP 5 -> 64 -> 64 -> 64 -> 3
 * with GELU, BF16 weights and activations, FP32 accumulation, its loss gradient and the AdamW
 * update.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA closure kernels (forward values, gradients,
 * optimiser step).  The closure has no counterpart in the reference; what it must reproduce is
 * the arithmetic stated here, step for step:
 *   - every operand of a product is rounded to BF16 (round to nearest even) -- inputs, weights,
 *     hidden activations, output gradients and pre-activation gradients, exactly the values the
 *     tensor cores read;
 *   - sums are FP32 (here: FP64, then compared with a tolerance, because the tensor core's
 *     summation order is its own);
 *   - biases are FP32 and added after the product; GELU is the erf form.
 *
 * Parameter layout (float, 8899): W1[64][5] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[3][64] b4[3].
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define NIN 5
#define NH 64
#define NOUT 3
#define OFF_W1 0
#define OFF_B1 (OFF_W1 + NH * NIN)
#define OFF_W2 (OFF_B1 + NH)
#define OFF_B2 (OFF_W2 + NH * NH)
#define OFF_W3 (OFF_B2 + NH)
#define OFF_B3 (OFF_W3 + NH * NH)
#define OFF_W4 (OFF_B3 + NH)
#define OFF_B4 (OFF_W4 + NOUT * NH)
#define NPARAM (OFF_B4 + NOUT)

int orc_closure_nparam(void) { return NPARAM; }

/* round to nearest even BF16, returned as float */
float orc_bf16(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  memcpy(&x, &u, 4);
  return x;
}

static float gelu(float a) { return 0.5f * a * (1.0f + erff(a * 0.70710678118654752f)); }

static float gelu_grad(float a) {
  return 0.5f * (1.0f + erff(a * 0.70710678118654752f)) + a * expf(-0.5f * a * a) * 0.39894228040143268f;
}

/* one layer: out[o] = sum_k in_b[k] * bf16(W[o][k]) (float sum, sequential) + b[o] */
static void layer(const float* P, int offW, int offB, int nout, int nin, const float* in_b, float* out) {
  for (int o = 0; o < nout; ++o) {
    float s = 0.0f;
    for (int k = 0; k < nin; ++k) s += in_b[k] * orc_bf16(P[offW + o * nin + k]);
    out[o] = s + P[offB + o];
  }
}

typedef struct {
  float xb[NIN];
  float a1[NH], a2[NH], a3[NH];
  float h1[NH], h2[NH], h3[NH];  /* BF16-rounded activations */
  float y[NOUT];
} fwd_state;

static void forward_one(const float* P, const float* x, fwd_state* s) {
  for (int k = 0; k < NIN; ++k) s->xb[k] = orc_bf16(x[k]);
  layer(P, OFF_W1, OFF_B1, NH, NIN, s->xb, s->a1);
  for (int k = 0; k < NH; ++k) s->h1[k] = orc_bf16(gelu(s->a1[k]));
  layer(P, OFF_W2, OFF_B2, NH, NH, s->h1, s->a2);
  for (int k = 0; k < NH; ++k) s->h2[k] = orc_bf16(gelu(s->a2[k]));
  layer(P, OFF_W3, OFF_B3, NH, NH, s->h2, s->a3);
  for (int k = 0; k < NH; ++k) s->h3[k] = orc_bf16(gelu(s->a3[k]));
  layer(P, OFF_W4, OFF_B4, NOUT, NH, s->h3, s->y);
}

/* y[n][3] = MLP(x[n][5]) */
void orc_closure_forward(const float* P, const float* x, int64_t n, float* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    fwd_state s;
    forward_one(P, x + i * NIN, &s);
    for (int o = 0; o < NOUT; ++o) y[i * NOUT + o] = s.y[o];
  }
}

/* Gradient of L = sum_i sum_o (y_io - t_io)^2 / n over the n points; grad has NPARAM entries. */
void orc_closure_grad(const float* P, const float* x, const float* t, int64_t n, double* grad, double* loss) {
  memset(grad, 0, sizeof(double) * NPARAM);
  double L = 0.0;
  const float inv = 1.0f / (float)n;
  for (int64_t i = 0; i < n; ++i) {
    fwd_state s;
    forward_one(P, x + i * NIN, &s);
    float dy[NOUT];
    for (int o = 0; o < NOUT; ++o) {
      const float e = s.y[o] - t[i * NOUT + o];
      L += (double)e * (double)e;
      dy[o] = orc_bf16(2.0f * e * inv);
    }
    /* layer 4 */
    float dh[NH], dz[NH];
    for (int o = 0; o < NOUT; ++o) {
      for (int k = 0; k < NH; ++k) grad[OFF_W4 + o * NH + k] += (double)dy[o] * s.h3[k];
      grad[OFF_B4 + o] += dy[o];
    }
    for (int k = 0; k < NH; ++k) {
      float a = 0.0f;
      for (int o = 0; o < NOUT; ++o) a += dy[o] * orc_bf16(P[OFF_W4 + o * NH + k]);
      dh[k] = a;
    }
    /* layer 3 */
    for (int k = 0; k < NH; ++k) dz[k] = orc_bf16(dh[k] * gelu_grad(s.a3[k]));
    for (int o = 0; o < NH; ++o) {
      for (int k = 0; k < NH; ++k) grad[OFF_W3 + o * NH + k] += (double)dz[o] * s.h2[k];
      grad[OFF_B3 + o] += dz[o];
    }
    for (int k = 0; k < NH; ++k) {
      float a = 0.0f;
      for (int o = 0; o < NH; ++o) a += dz[o] * orc_bf16(P[OFF_W3 + o * NH + k]);
      dh[k] = a;
    }
    /* layer 2 */
    for (int k = 0; k < NH; ++k) dz[k] = orc_bf16(dh[k] * gelu_grad(s.a2[k]));
    for (int o = 0; o < NH; ++o) {
      for (int k = 0; k < NH; ++k) grad[OFF_W2 + o * NH + k] += (double)dz[o] * s.h1[k];
      grad[OFF_B2 + o] += dz[o];
    }
    for (int k = 0; k < NH; ++k) {
      float a = 0.0f;
      for (int o = 0; o < NH; ++o) a += dz[o] * orc_bf16(P[OFF_W2 + o * NH + k]);
      dh[k] = a;
    }
    /* layer 1 */
    for (int k = 0; k < NH; ++k) dz[k] = orc_bf16(dh[k] * gelu_grad(s.a1[k]));
    for (int o = 0; o < NH; ++o) {
      for (int k = 0; k < NIN; ++k) grad[OFF_W1 + o * NIN + k] += (double)dz[o] * s.xb[k];
      grad[OFF_B1 + o] += dz[o];
    }
  }
  *loss = L / (double)n;
}

/* One AdamW step (decoupled weight decay on the weight matrices only), step number t >= 1. */
void orc_closure_adamw(float* P, float* m, float* v, const float* g, int t, float lr, float b1, float b2, float eps,
                       float wd) {
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  for (int i = 0; i < NPARAM; ++i) {
    const int is_bias = (i >= OFF_B1 && i < OFF_W2) || (i >= OFF_B2 && i < OFF_W3) || (i >= OFF_B3 && i < OFF_W4) ||
                        i >= OFF_B4;
    m[i] = b1 * m[i] + (1.0f - b1) * g[i];
    v[i] = b2 * v[i] + (1.0f - b2) * g[i] * g[i];
    const float mh = m[i] / c1, vh = v[i] / c2;
    float p = P[i];
    if (!is_bias) p -= lr * wd * p;
    P[i] = p - lr * mh / (sqrtf(vh) + eps);
  }
}
