/*
 * mlp_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU forward and backward pass of the learned property model (1 -> 64 ->
 * 64 -> 6 tanh MLP from rho*h to the outputs of THERM_PROP_UPDATE_FROM_DH),
 * the checker of the tensor-core training and inference kernels.  The GPU
 * rounds the operands of its tensor-core products to BF16 (the weights of
 * layers 2 and 3, the activations h1 and h2, and the hidden-layer error dz2)
 * and accumulates in FP32; here the same values are rounded to BF16 (round
 * to nearest even) and the sums are taken in FP64.  Element-wise steps use
 * the GPU's FP32 operations (fmaf, tanhf).  The inference form rounds each
 * hidden activation's input and result to FP16, as the GPU's paired
 * activation does, and its tensor-core operands are FP16 (the activations as
 * they come out of the activation, the weights rounded to FP16).  Targets come from the table
 * search of thermo_oracle.c, bitwise equal to the GPU's.
 *
 * Parameter layout (FP32): w1[64], b1[64], W2[64][64] (out, in), b2[64],
 * W3[6][64], b3[6].  norm: x_lo, x_hi, off[6], scale[6].
 *
 * Activation (orc_mlp_set_activation): 0 tanh, 1 the clamped cubic
 * c = clamp(z, -1, 1), h = c (3 - c^2) / 2, h' = 3 (1 - c^2) / 2, evaluated in
 * the GPU's operation order (FP32 for training; FP16 pair arithmetic for
 * inference, each product rounded to FP16 and the multiply-add rounded once).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define H 64
#define NO 6
#define P_W1 0
#define P_B1 (P_W1 + H)
#define P_W2 (P_B1 + H)
#define P_B2 (P_W2 + H * H)
#define P_W3 (P_B2 + H)
#define P_B3 (P_W3 + NO * H)
#define NPARAM (P_B3 + NO)

int orc_prop_point(void* tab, double dh, double* out);

static float bf16r(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return f;
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&f, &u, 4);
    return f;
}

/* Round to FP16 (round to nearest even) and back: inference evaluates each
 * hidden activation as a pair instruction on FP16 operands (the GPU's
 * tanh.approx.f16x2), so its input and its result are FP16 values. */
static float f16r(float f) { return (float)(_Float16)f; }

static int g_act = 0;
void orc_mlp_set_activation(int act) { g_act = act ? 1 : 0; }

static float act_f(float z) {
    if (!g_act) return tanhf(z);
    const float c = z < -1.f ? -1.f : (z > 1.f ? 1.f : z);
    return c * (1.5f - 0.5f * c * c);
}
static float act_d(float z, float h) {
    if (!g_act) return 1.f - h * h;
    const float c = z < -1.f ? -1.f : (z > 1.f ? 1.f : z);
    return 1.5f * (1.f - c * c);
}
/* inference form on an FP16 pre-activation: the GPU's tanh.approx.f16x2 (emulated by the exact
 * tanh rounded to FP16) or the clamped cubic in FP16 pair arithmetic */
static float act_inf(float pre) {
    if (!g_act) return f16r(tanhf(pre));
    const float c = pre < -1.f ? -1.f : (pre > 1.f ? 1.f : pre);
    const float c2 = f16r(c * c);                                   /* exact product, one rounding */
    const float s = (float)(_Float16)((double)c2 * -0.5 + 1.5);      /* fused: one rounding */
    return f16r(c * s);
}

static float xnorm(const double* norm, double dh) {
    const double lo = (double)(float)norm[0], hi = (double)(float)norm[1];
    return (float)(2.0 * (dh - lo) / (hi - lo) - 1.0);
}

static void forward(const float* p, float x, float* h1, float* h2, float* z2, float* y) {
    for (int i = 0; i < H; ++i) h1[i] = act_f(fmaf(p[P_W1 + i], x, p[P_B1 + i]));
    for (int j = 0; j < H; ++j) {
        double a = 0.0;
        for (int i = 0; i < H; ++i) a += (double)bf16r(h1[i]) * (double)bf16r(p[P_W2 + j * H + i]);
        z2[j] = (float)a + p[P_B2 + j];
        h2[j] = act_f(z2[j]);
    }
    for (int k = 0; k < NO; ++k) {
        double a = 0.0;
        for (int j = 0; j < H; ++j) a += (double)bf16r(h2[j]) * (double)bf16r(p[P_W3 + k * H + j]);
        y[k] = (float)a + p[P_B3 + k];
    }
}

/* The inference form of forward(): the FP16 rounding of every hidden
 * activation's input and result, with the exact tanh in between (the GPU's
 * hardware tanh adds its own approximation, about 2^-11 relative), the first
 * layer's pre-activation in FP16 fused multiply-adds, and FP16 operands of the
 * two tensor-core products (h1 and h2 are FP16 values already; W2 and W3 are
 * rounded to FP16). */
static void forward_inf(const float* p, float x, float* h1, float* h2, float* y) {
    /* first layer in FP16 arithmetic: x = xh + xl, pre = fma(w1, xh, fma(w1, xl, b1)), each fma
     * rounded once to FP16 (the products and sums of FP16 values are exact in FP64) */
    const float xh = f16r(x), xl = f16r(x - xh);
    for (int i = 0; i < H; ++i) {
        const double w = (double)f16r(p[P_W1 + i]), b = (double)f16r(p[P_B1 + i]);
        const double inner = (double)(_Float16)(w * (double)xl + b);
        const float pre = (float)(_Float16)(w * (double)xh + inner);
        h1[i] = act_inf(pre);
    }
    for (int j = 0; j < H; ++j) {
        double a = 0.0;
        for (int i = 0; i < H; ++i) a += (double)h1[i] * (double)f16r(p[P_W2 + j * H + i]);
        h2[j] = act_inf(f16r((float)a + p[P_B2 + j]));
    }
    for (int k = 0; k < NO; ++k) {
        double a = 0.0;
        for (int j = 0; j < H; ++j) a += (double)h2[j] * (double)f16r(p[P_W3 + k * H + j]);
        y[k] = (float)a + p[P_B3 + k];
    }
}

/* Model outputs (denormalised) for n points, as inference evaluates them:
 * out[6n] in the order H, T, D, M, K, CP. */
void orc_mlp_forward(const float* p, const double* norm, int n, const double* dh, double* out) {
    float h1[H], h2[H], y[NO];
    for (int q = 0; q < n; ++q) {
        forward_inf(p, xnorm(norm, dh[q]), h1, h2, y);
        for (int k = 0; k < NO; ++k) out[(size_t)k * n + q] = (double)((float)norm[2 + k] + (float)norm[2 + NO + k] * y[k]);
    }
}

/* Gradient of the mean squared error over n samples and 6 normalised outputs
 * (targets from the table search).  grad[NPARAM]; returns the loss, or -1
 * when a sample lies outside the table. */
double orc_mlp_gradients(void* tab, const float* p, const double* norm, int n, const double* dh, double* grad) {
    memset(grad, 0, sizeof(double) * NPARAM);
    const float inv = 1.0f / ((float)n * NO);
    double loss = 0.0;
    static double dW2[H * H];
    memset(dW2, 0, sizeof(dW2));
    for (int q = 0; q < n; ++q) {
        double o[6];
        if (orc_prop_point(tab, dh[q], o)) return -1.0;
        const float x = xnorm(norm, dh[q]);
        float h1[H], h2[H], z2[H], y[NO], dy[NO], dz2[H];
        forward(p, x, h1, h2, z2, y);
        for (int k = 0; k < NO; ++k) {
            const float t = (float)((o[k] - (double)(float)norm[2 + k]) / (double)(float)norm[2 + NO + k]);
            const float e = y[k] - t;
            loss += (double)(e * e * inv);
            dy[k] = 2.f * e * inv;
            grad[P_B3 + k] += dy[k];
        }
        for (int j = 0; j < H; ++j) {
            float s = 0.f;
            for (int k = 0; k < NO; ++k) {
                s = fmaf(dy[k], p[P_W3 + k * H + j], s);
                grad[P_W3 + k * H + j] += (double)(dy[k] * h2[j]);
            }
            dz2[j] = s * act_d(z2[j], h2[j]);
            grad[P_B2 + j] += dz2[j];
        }
        for (int i = 0; i < H; ++i) {
            double a = 0.0;
            for (int j = 0; j < H; ++j) a += (double)bf16r(dz2[j]) * (double)bf16r(p[P_W2 + j * H + i]);
            const float dz1 = (float)a * act_d(fmaf(p[P_W1 + i], x, p[P_B1 + i]), h1[i]);
            grad[P_W1 + i] += (double)(dz1 * x);
            grad[P_B1 + i] += dz1;
        }
        for (int j = 0; j < H; ++j)
            for (int i = 0; i < H; ++i) dW2[j * H + i] += (double)bf16r(dz2[j]) * (double)bf16r(h1[i]);
    }
    for (int q = 0; q < H * H; ++q) grad[P_W2 + q] = dW2[q];
    return loss;
}
