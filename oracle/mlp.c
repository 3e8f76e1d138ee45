/*
 * CPU oracle of the learned block-Jacobi correction (TEST INFRASTRUCTURE ONLY).
 *
 * The reference has no learned preconditioner: this is the FP64 restatement the device
 * kernels of plamatrix_b200 are checked against, itself pinned by finite differences in
 * tests/test_mlp_oracle.py.  Definitions (shared with the device code):
 *
 *   features (25 per block row p of the reduced system S, with s = mean diag(S_pp), or 1
 *   when that mean is not positive):
 *     f[k], k = r(r+1)/2 + c (c <= r):  a = S_pp[r][c] / s,  f = sign(a) log1p(|a|)
 *     f[21..23] = log1p(mean), log1p(max), log1p(min) of ||S_pq||_F / s over q != p
 *     f[24]     = log1p(number of such blocks) / 4          (all zero without any)
 *   network: z1 = f W1 + b1, h1 = gelu(z1), z2 = h1 W2 + b2, h2 = gelu(z2), o = h2 W3 + b3,
 *     25 -> 128 -> 128 -> 21, gelu(x) = x Phi(x); W stored input-major (W[k][n]).
 *   correction of the block-Jacobi Cholesky factor L (S_pp = L L^T, symmetrised from its lower
 *   triangle), o indexed like f[0..20]:
 *     L'_ii = L_ii softplus(o_ii) / ln 2,   L'_ij = L_ij + o_ij L_jj  (i > j)
 *   preconditioner block M_p = L' L'^T (SPD); o = 0 gives back block Jacobi.
 *   training loss of a system with solution x and right-hand side b (b = S x):
 *     loss = sum_p ||M_p x_p - b_p||^2 / sum_p ||b_p||^2
 *
 * With `bf16` set, GEMM operands (features, hidden activations, weights) are rounded to
 * bfloat16 (round to nearest even) before the products, as the device does; sums stay FP64.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

#define IN ORC_MLP_IN
#define HID ORC_MLP_HIDDEN
#define OUT ORC_MLP_OUT

static double bf16(double v)
{
    float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) != 0x7f800000u)
    {
        const uint32_t lsb = (u >> 16) & 1u;
        u += 0x7fffu + lsb;
    }
    u &= 0xffff0000u;
    memcpy(&f, &u, 4);
    return (double)f;
}

static double gelu(double x) { return 0.5 * x * (1.0 + erf(x / sqrt(2.0))); }
static double gelu_grad(double x)
{
    return 0.5 * (1.0 + erf(x / sqrt(2.0))) + x * exp(-0.5 * x * x) / sqrt(2.0 * M_PI);
}
static double softplus(double x) { return x > 30.0 ? x : log1p(exp(x)); }
static double sigmoid(double x) { return 1.0 / (1.0 + exp(-x)); }

/* offsets of the flat parameter vector */
#define OFF_W1 0
#define OFF_B1 (OFF_W1 + IN * HID)
#define OFF_W2 (OFF_B1 + HID)
#define OFF_B2 (OFF_W2 + HID * HID)
#define OFF_W3 (OFF_B2 + HID)
#define OFF_B3 (OFF_W3 + HID * OUT)

int64_t orc_mlp_param_count(void) { return OFF_B3 + OUT; }

int orc_mlp_features(int64_t P, const int64_t* block_row_ptr, const int64_t* block_col, const double* blocks,
                     double* features)
{
    for (int64_t p = 0; p < P; ++p)
    {
        const double* d = NULL;
        double sum = 0.0, mx = 0.0, mn = 0.0;
        int64_t n = 0;
        for (int64_t b = block_row_ptr[p]; b < block_row_ptr[p + 1]; ++b)
            if (block_col[b] == p)
                d = blocks + b * 36;
        if (!d)
            return ORC_INVALID_ARGUMENT;
        double s = 0.0;
        for (int i = 0; i < 6; ++i)
            s += d[i * 6 + i];
        s /= 6.0;
        if (!(s > 0.0))
            s = 1.0;
        double* f = features + p * IN;
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c <= r; ++c)
            {
                const double a = d[r * 6 + c] / s;
                f[r * (r + 1) / 2 + c] = (a < 0.0 ? -1.0 : 1.0) * log1p(fabs(a));
            }
        for (int64_t b = block_row_ptr[p]; b < block_row_ptr[p + 1]; ++b)
        {
            if (block_col[b] == p)
                continue;
            double fro = 0.0;
            for (int k = 0; k < 36; ++k)
                fro += blocks[b * 36 + k] * blocks[b * 36 + k];
            fro = sqrt(fro) / s;
            sum += fro;
            mx = n == 0 || fro > mx ? fro : mx;
            mn = n == 0 || fro < mn ? fro : mn;
            ++n;
        }
        f[21] = n ? log1p(sum / (double)n) : 0.0;
        f[22] = n ? log1p(mx) : 0.0;
        f[23] = n ? log1p(mn) : 0.0;
        f[24] = log1p((double)n) / 4.0;
    }
    return ORC_OK;
}

/* caches: z1, h1, z2, h2 (P x HID each) may be NULL when not needed */
int orc_mlp_forward(int64_t P, const double* features, const double* params, int bf16_operands, double* z1,
                    double* h1, double* z2, double* h2, double* out)
{
    const double* W1 = params + OFF_W1;
    const double* B1 = params + OFF_B1;
    const double* W2 = params + OFF_W2;
    const double* B2 = params + OFF_B2;
    const double* W3 = params + OFF_W3;
    const double* B3 = params + OFF_B3;
    double a[HID], g1[HID], g2[HID];
#define Q(v) (bf16_operands ? bf16(v) : (v))
    for (int64_t p = 0; p < P; ++p)
    {
        const double* f = features + p * IN;
        for (int n = 0; n < HID; ++n)
        {
            double s = 0.0;
            for (int k = 0; k < IN; ++k)
                s += Q(f[k]) * Q(W1[k * HID + n]);
            a[n] = s + B1[n];
            g1[n] = gelu(a[n]);
            if (z1)
                z1[p * HID + n] = a[n];
            if (h1)
                h1[p * HID + n] = g1[n];
        }
        for (int n = 0; n < HID; ++n)
        {
            double s = 0.0;
            for (int k = 0; k < HID; ++k)
                s += Q(g1[k]) * Q(W2[k * HID + n]);
            a[n] = s + B2[n];
            g2[n] = gelu(a[n]);
            if (z2)
                z2[p * HID + n] = a[n];
            if (h2)
                h2[p * HID + n] = g2[n];
        }
        for (int n = 0; n < OUT; ++n)
        {
            double s = 0.0;
            for (int k = 0; k < HID; ++k)
                s += Q(g2[k]) * Q(W3[k * OUT + n]);
            out[p * OUT + n] = s + B3[n];
        }
    }
#undef Q
    return ORC_OK;
}

/* Cholesky factor of the symmetrised lower triangle of a 6x6 block; 0 when not SPD */
static int chol6(const double* d, double* L)
{
    memset(L, 0, 36 * sizeof(double));
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j <= i; ++j)
        {
            double v = d[i * 6 + j];
            for (int k = 0; k < j; ++k)
                v -= L[i * 6 + k] * L[j * 6 + k];
            if (i == j)
            {
                if (!(v > 0.0))
                    return 0;
                L[i * 6 + i] = sqrt(v);
            }
            else
            {
                L[i * 6 + j] = v / L[j * 6 + j];
            }
        }
    return 1;
}

static void corrected(const double* L, const double* o, double* Lc)
{
    memset(Lc, 0, 36 * sizeof(double));
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j <= i; ++j)
        {
            const double oo = o[i * (i + 1) / 2 + j];
            Lc[i * 6 + j] = i == j ? L[i * 6 + i] * softplus(oo) / log(2.0) : L[i * 6 + j] + oo * L[j * 6 + j];
        }
}

int orc_mlp_loss_grad(int64_t P, const double* diag_blocks, const double* out, const double* x, const double* b,
                      double* loss, double* dout)
{
    double num = 0.0, den = 0.0;
    for (int64_t p = 0; p < P; ++p)
        for (int i = 0; i < 6; ++i)
            den += b[p * 6 + i] * b[p * 6 + i];
    if (!(den > 0.0))
        return ORC_INVALID_ARGUMENT;
    for (int64_t p = 0; p < P; ++p)
    {
        double L[36], Lc[36], u[6], r[6], v[6];
        if (!chol6(diag_blocks + p * 36, L))
            return ORC_RUNTIME_ERROR;
        const double* o = out + p * OUT;
        corrected(L, o, Lc);
        const double* xp = x + p * 6;
        for (int j = 0; j < 6; ++j)
        {
            u[j] = 0.0;
            for (int i = j; i < 6; ++i)
                u[j] += Lc[i * 6 + j] * xp[i];
        }
        for (int i = 0; i < 6; ++i)
        {
            double s = 0.0;
            for (int j = 0; j <= i; ++j)
                s += Lc[i * 6 + j] * u[j];
            r[i] = s - b[p * 6 + i];
            num += r[i] * r[i];
        }
        for (int j = 0; j < 6; ++j)
        {
            v[j] = 0.0;
            for (int i = j; i < 6; ++i)
                v[j] += Lc[i * 6 + j] * r[i];
        }
        if (dout)
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j <= i; ++j)
                {
                    const int k = i * (i + 1) / 2 + j;
                    const double g = 2.0 * (r[i] * u[j] + xp[i] * v[j]) / den;
                    dout[p * OUT + k] =
                        i == j ? g * L[i * 6 + i] * sigmoid(o[k]) / log(2.0) : g * L[j * 6 + j];
                }
    }
    *loss = num / den;
    return ORC_OK;
}

/* Probe loss of the preconditioned operator: sum_p ||v_p - A_p^-1 u_p||^2 / ||v||^2 with
 * A_p = L'_p L'_p^T and u = S v supplied; analytic gradient with respect to the outputs
 * (derivation: w = A^-1 u, e = v - w, d loss = 2 (A^-1 e)^T dA w / den, dA = dL' L'^T + L' dL'^T). */
static void lsolve6(const double* L, const double* b, double* x)
{
    for (int i = 0; i < 6; ++i)
    {
        double s = b[i];
        for (int j = 0; j < i; ++j)
            s -= L[i * 6 + j] * x[j];
        x[i] = s / L[i * 6 + i];
    }
}

static void usolve6(const double* L, const double* b, double* x)
{
    for (int i = 5; i >= 0; --i)
    {
        double s = b[i];
        for (int j = i + 1; j < 6; ++j)
            s -= L[j * 6 + i] * x[j];
        x[i] = s / L[i * 6 + i];
    }
}

int orc_mlp_probe_loss_grad(int64_t P, const double* diag_blocks, const double* out, const double* v, const double* sv,
                            double* loss, double* dout)
{
    double num = 0.0, den = 0.0;
    for (int64_t p = 0; p < P; ++p)
        for (int i = 0; i < 6; ++i)
            den += v[p * 6 + i] * v[p * 6 + i];
    if (!(den > 0.0))
        return ORC_INVALID_ARGUMENT;
    for (int64_t p = 0; p < P; ++p)
    {
        double L[36], Lc[36], y[6], w[6], e[6], z[6], q[6];
        if (!chol6(diag_blocks + p * 36, L))
            return ORC_RUNTIME_ERROR;
        const double* o = out + p * OUT;
        corrected(L, o, Lc);
        lsolve6(Lc, sv + p * 6, y);
        usolve6(Lc, y, w);
        for (int i = 0; i < 6; ++i)
        {
            e[i] = v[p * 6 + i] - w[i];
            num += e[i] * e[i];
        }
        lsolve6(Lc, e, z);
        usolve6(Lc, z, q);
        if (dout)
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j <= i; ++j)
                {
                    const int k = i * (i + 1) / 2 + j;
                    const double g = 2.0 * (q[i] * y[j] + w[i] * z[j]) / den;
                    dout[p * OUT + k] =
                        i == j ? g * L[i * 6 + i] * sigmoid(o[k]) / log(2.0) : g * L[j * 6 + j];
                }
    }
    *loss = num / den;
    return ORC_OK;
}

int orc_mlp_backward(int64_t P, const double* features, const double* params, int bf16_operands, const double* z1,
                     const double* h1, const double* z2, const double* h2, const double* dout, double* grads)
{
    const double* W2 = params + OFF_W2;
    const double* W3 = params + OFF_W3;
    const int64_t n = orc_mlp_param_count();
    for (int64_t k = 0; k < n; ++k)
        grads[k] = 0.0;
    double* dW1 = grads + OFF_W1;
    double* dB1 = grads + OFF_B1;
    double* dW2 = grads + OFF_W2;
    double* dB2 = grads + OFF_B2;
    double* dW3 = grads + OFF_W3;
    double* dB3 = grads + OFF_B3;
    double dz2[HID], dz1[HID];
#define Q(v) (bf16_operands ? bf16(v) : (v))
    for (int64_t p = 0; p < P; ++p)
    {
        const double* d = dout + p * OUT;
        for (int k = 0; k < HID; ++k)
        {
            double s = 0.0;
            for (int m = 0; m < OUT; ++m)
                s += Q(d[m]) * Q(W3[k * OUT + m]);
            dz2[k] = s * gelu_grad(z2[p * HID + k]);
        }
        for (int k = 0; k < HID; ++k)
        {
            double s = 0.0;
            for (int m = 0; m < HID; ++m)
                s += Q(dz2[m]) * Q(W2[k * HID + m]);
            dz1[k] = s * gelu_grad(z1[p * HID + k]);
        }
        for (int k = 0; k < HID; ++k)
            for (int m = 0; m < OUT; ++m)
                dW3[k * OUT + m] += Q(h2[p * HID + k]) * Q(d[m]);
        for (int m = 0; m < OUT; ++m)
            dB3[m] += d[m];
        for (int k = 0; k < HID; ++k)
            for (int m = 0; m < HID; ++m)
                dW2[k * HID + m] += Q(h1[p * HID + k]) * Q(dz2[m]);
        for (int m = 0; m < HID; ++m)
            dB2[m] += dz2[m];
        for (int k = 0; k < IN; ++k)
            for (int m = 0; m < HID; ++m)
                dW1[k * HID + m] += Q(features[p * IN + k]) * Q(dz1[m]);
        for (int m = 0; m < HID; ++m)
            dB1[m] += dz1[m];
    }
#undef Q
    return ORC_OK;
}

int orc_mlp_preconditioner(int64_t P, const double* diag_blocks, const double* out, double* minv)
{
    for (int64_t p = 0; p < P; ++p)
    {
        double L[36], Lc[36], M[36];
        if (!chol6(diag_blocks + p * 36, L))
            return ORC_RUNTIME_ERROR;
        corrected(L, out + p * OUT, Lc);
        /* inverse of L' L'^T: columns e_c -> forward then backward substitution */
        for (int c = 0; c < 6; ++c)
        {
            double y[6];
            for (int i = 0; i < 6; ++i)
            {
                double v = i == c ? 1.0 : 0.0;
                for (int k = 0; k < i; ++k)
                    v -= Lc[i * 6 + k] * y[k];
                y[i] = v / Lc[i * 6 + i];
            }
            for (int i = 5; i >= 0; --i)
            {
                double v = y[i];
                for (int k = i + 1; k < 6; ++k)
                    v -= Lc[k * 6 + i] * M[k * 6 + c];
                M[i * 6 + c] = v / Lc[i * 6 + i];
            }
        }
        memcpy(minv + p * 36, M, sizeof(M));
    }
    return ORC_OK;
}
