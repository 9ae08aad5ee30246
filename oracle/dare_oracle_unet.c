/*
 * dare_oracle_unet.c -- CPU restatement of the learned linear preconditioner
 * N(u) = u + U(u) (forward pass, loss, analytic gradient).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the tcgen05 convolution kernels
 * of dare_b200 (forward, data gradient, weight gradient, level transfers,
 * loss).  Nothing in the product links it.
 *
 * The reference has no learned preconditioner (DaRe's BiCGStab2 takes the
 * Jacobi preconditioner only, BiCGStab2.inl:258-261), so there is no reference
 * code to pin this against; it is pinned instead by its own finite-difference
 * check (the loss is quadratic in every single weight, so a central
 * difference is exact up to rounding) and the GPU kernels are checked
 * against it.
 *
 * Network (all bias-free and activation-free):
 *   enc0 = conv(u; 1->16)                      level 0 (n)
 *   p1 = avgpool(enc0); enc1 = conv(p1; 16->32) level 1 (n/2)
 *   p2 = avgpool(enc1); enc2 = conv(p2; 32->64) level 2
 *   p3 = avgpool(enc2); e3 = conv(p3; 64->64)   level 3
 *   s2 = enc2 + up(conv(e3; 64->64))            (dec3)
 *   s1 = enc1 + up(conv(s2; 64->32))            (dec2)
 *   s0 = enc0 + up(conv(s1; 32->16))            (dec1)
 *   z  = u + conv(s0; 16->1)                    (dec0)
 * conv: 3x3x3, zero padding, out[p][o] = sum_t sum_i W[t][o][i] in[p + d_t][i],
 * d_t = (t/9 - 1, (t/3)%3 - 1, t%3 - 1); avgpool: mean of the 2x2x2
 * children; up: nearest-neighbour copy to the 8 children.
 * With `bf16` set, every stored activation and gradient tensor, the weights
 * and the network input are rounded to bfloat16 (round to nearest even) at
 * the points where the GPU stores them; the arithmetic stays in double.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "dare_oracle_unet.h"

static const int kCin[8] = {1, 16, 32, 64, 64, 64, 32, 16};
static const int kCout[8] = {16, 32, 64, 64, 64, 32, 16, 1};

static double rb(double x) {
    float f = (float)x;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return (double)f; /* inf / nan */
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    memcpy(&f, &u, 4);
    return (double)f;
}

typedef struct {
    int n[3];
    int64_t cells;
} Lev;

static void round_all(double* a, int64_t m, int on) {
    if (!on) return;
    for (int64_t i = 0; i < m; i++) a[i] = rb(a[i]);
}

/* out[p][o] (+)= sum_t sum_i W[t][o][i] in[p + d_t][i] */
static void conv(const Lev* L, const double* in, int cin, const double* W, int cout, double* out) {
    const int n0 = L->n[0], n1 = L->n[1], n2 = L->n[2];
    memset(out, 0, sizeof(double) * (size_t)L->cells * cout);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
            for (int k = 0; k < n2; k++) {
                double* o = out + (((int64_t)i * n1 + j) * n2 + k) * cout;
                for (int t = 0; t < 27; t++) {
                    const int ii = i + t / 9 - 1, jj = j + (t / 3) % 3 - 1, kk = k + t % 3 - 1;
                    if (ii < 0 || ii >= n0 || jj < 0 || jj >= n1 || kk < 0 || kk >= n2) continue;
                    const double* x = in + (((int64_t)ii * n1 + jj) * n2 + kk) * cin;
                    const double* w = W + (int64_t)t * cout * cin;
                    for (int a = 0; a < cout; a++) {
                        double s = 0.;
                        for (int b = 0; b < cin; b++) s += w[a * cin + b] * x[b];
                        o[a] += s;
                    }
                }
            }
}

/* data gradient: dx[q][i] = sum_t sum_o W[t][o][i] dy[q - d_t][o] */
static void conv_t(const Lev* L, const double* dy, int cout, const double* W, int cin, double* dx) {
    const int n0 = L->n[0], n1 = L->n[1], n2 = L->n[2];
    memset(dx, 0, sizeof(double) * (size_t)L->cells * cin);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
            for (int k = 0; k < n2; k++) {
                double* o = dx + (((int64_t)i * n1 + j) * n2 + k) * cin;
                for (int t = 0; t < 27; t++) {
                    const int ii = i - (t / 9 - 1), jj = j - ((t / 3) % 3 - 1), kk = k - (t % 3 - 1);
                    if (ii < 0 || ii >= n0 || jj < 0 || jj >= n1 || kk < 0 || kk >= n2) continue;
                    const double* g = dy + (((int64_t)ii * n1 + jj) * n2 + kk) * cout;
                    const double* w = W + (int64_t)t * cout * cin;
                    for (int b = 0; b < cin; b++) {
                        double s = 0.;
                        for (int a = 0; a < cout; a++) s += w[a * cin + b] * g[a];
                        o[b] += s;
                    }
                }
            }
}

/* weight gradient: gW[t][o][i] += scale * sum_p dy[p][o] x[p + d_t][i] */
static void conv_w(const Lev* L, const double* x, int cin, const double* dy, int cout, double scale, double* gW) {
    const int n0 = L->n[0], n1 = L->n[1], n2 = L->n[2];
#pragma omp parallel for schedule(static)
    for (int t = 0; t < 27; t++) {
        const int di = t / 9 - 1, dj = (t / 3) % 3 - 1, dk = t % 3 - 1;
        double* acc = (double*)calloc((size_t)cout * cin, sizeof(double));
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++)
                for (int k = 0; k < n2; k++) {
                    const int ii = i + di, jj = j + dj, kk = k + dk;
                    if (ii < 0 || ii >= n0 || jj < 0 || jj >= n1 || kk < 0 || kk >= n2) continue;
                    const double* g = dy + (((int64_t)i * n1 + j) * n2 + k) * cout;
                    const double* xx = x + (((int64_t)ii * n1 + jj) * n2 + kk) * cin;
                    for (int a = 0; a < cout; a++)
                        for (int b = 0; b < cin; b++) acc[a * cin + b] += g[a] * xx[b];
                }
        for (int m = 0; m < cout * cin; m++) gW[(int64_t)t * cout * cin + m] += scale * acc[m];
        free(acc);
    }
}

/* coarse = scale * sum of the 8 children */
static void restrict2(const Lev* F, const Lev* Cl, const double* fine, int c, double scale, double* coarse) {
    for (int i = 0; i < Cl->n[0]; i++)
        for (int j = 0; j < Cl->n[1]; j++)
            for (int k = 0; k < Cl->n[2]; k++) {
                double* o = coarse + (((int64_t)i * Cl->n[1] + j) * Cl->n[2] + k) * c;
                for (int ch = 0; ch < c; ch++) o[ch] = 0.;
                for (int q = 0; q < 8; q++) {
                    const int fi = 2 * i + (q >> 2), fj = 2 * j + ((q >> 1) & 1), fk = 2 * k + (q & 1);
                    const double* f = fine + (((int64_t)fi * F->n[1] + fj) * F->n[2] + fk) * c;
                    for (int ch = 0; ch < c; ch++) o[ch] += f[ch];
                }
                for (int ch = 0; ch < c; ch++) o[ch] *= scale;
            }
}

/* fine[child] = fine[child] + scale * coarse[parent] (rounded if bf) */
static void prolong_add(const Lev* F, const Lev* Cl, const double* coarse, int c, double scale, double* fine, int bf) {
    for (int i = 0; i < F->n[0]; i++)
        for (int j = 0; j < F->n[1]; j++)
            for (int k = 0; k < F->n[2]; k++) {
                double* f = fine + (((int64_t)i * F->n[1] + j) * F->n[2] + k) * c;
                const double* q = coarse + (((int64_t)(i / 2) * Cl->n[1] + j / 2) * Cl->n[2] + k / 2) * c;
                for (int ch = 0; ch < c; ch++) f[ch] = bf ? rb(f[ch] + scale * q[ch]) : f[ch] + scale * q[ch];
            }
}

int64_t dor_unet_num_params(void) {
    int64_t s = 0;
    for (int l = 0; l < 8; l++) s += 27LL * kCin[l] * kCout[l];
    return s;
}

typedef struct {
    Lev lv[4];
    double* Wl[8];
    double* S0; double* P1; double* S1; double* P2; double* S2; double* P3; double* E3;
    double* x0;   /* network input as the first conv sees it */
    double* tmp;
} Net;

static int net_init(Net* N, const int n[3], const float* w, int bf) {
    memset(N, 0, sizeof(*N));
    for (int d = 0; d < 3; d++)
        if (n[d] < 8 || n[d] % 8) return -1;
    for (int l = 0; l < 4; l++) {
        for (int d = 0; d < 3; d++) N->lv[l].n[d] = n[d] >> l;
        N->lv[l].cells = (int64_t)N->lv[l].n[0] * N->lv[l].n[1] * N->lv[l].n[2];
    }
    int64_t off = 0;
    for (int l = 0; l < 8; l++) {
        const int64_t m = 27LL * kCin[l] * kCout[l];
        N->Wl[l] = (double*)malloc(sizeof(double) * m);
        for (int64_t i = 0; i < m; i++) N->Wl[l][i] = bf ? rb(w[off + i]) : (double)w[off + i];
        off += m;
    }
    const int64_t c0 = N->lv[0].cells, c1 = N->lv[1].cells, c2 = N->lv[2].cells, c3 = N->lv[3].cells;
    N->S0 = (double*)malloc(sizeof(double) * c0 * 16);
    N->P1 = (double*)malloc(sizeof(double) * c1 * 16);
    N->S1 = (double*)malloc(sizeof(double) * c1 * 32);
    N->P2 = (double*)malloc(sizeof(double) * c2 * 32);
    N->S2 = (double*)malloc(sizeof(double) * c2 * 64);
    N->P3 = (double*)malloc(sizeof(double) * c3 * 64);
    N->E3 = (double*)malloc(sizeof(double) * c3 * 64);
    N->x0 = (double*)malloc(sizeof(double) * c0);
    N->tmp = (double*)malloc(sizeof(double) * c0 * 64);
    return 0;
}

static void net_free(Net* N) {
    for (int l = 0; l < 8; l++) free(N->Wl[l]);
    free(N->S0); free(N->P1); free(N->S1); free(N->P2); free(N->S2); free(N->P3); free(N->E3);
    free(N->x0); free(N->tmp);
}

/* forward; z over the level-0 cells */
static void net_forward(Net* N, const double* u, int bf, double* z) {
    const Lev* L = N->lv;
    double* t = N->tmp;
    for (int64_t c = 0; c < L[0].cells; c++) N->x0[c] = bf ? rb(u[c]) : u[c];
    conv(&L[0], N->x0, 1, N->Wl[0], 16, N->S0);
    round_all(N->S0, L[0].cells * 16, bf);
    restrict2(&L[0], &L[1], N->S0, 16, 0.125, N->P1);
    round_all(N->P1, L[1].cells * 16, bf);
    conv(&L[1], N->P1, 16, N->Wl[1], 32, N->S1);
    round_all(N->S1, L[1].cells * 32, bf);
    restrict2(&L[1], &L[2], N->S1, 32, 0.125, N->P2);
    round_all(N->P2, L[2].cells * 32, bf);
    conv(&L[2], N->P2, 32, N->Wl[2], 64, N->S2);
    round_all(N->S2, L[2].cells * 64, bf);
    restrict2(&L[2], &L[3], N->S2, 64, 0.125, N->P3);
    round_all(N->P3, L[3].cells * 64, bf);
    conv(&L[3], N->P3, 64, N->Wl[3], 64, N->E3);
    round_all(N->E3, L[3].cells * 64, bf);
    conv(&L[3], N->E3, 64, N->Wl[4], 64, t);               /* dec3 */
    prolong_add(&L[2], &L[3], t, 64, 1.0, N->S2, bf);
    conv(&L[2], N->S2, 64, N->Wl[5], 32, t);               /* dec2 */
    prolong_add(&L[1], &L[2], t, 32, 1.0, N->S1, bf);
    conv(&L[1], N->S1, 32, N->Wl[6], 16, t);               /* dec1 */
    round_all(t, L[1].cells * 16, bf);                     /* stored at level 1, then added */
    prolong_add(&L[0], &L[1], t, 16, 1.0, N->S0, bf);
    conv(&L[0], N->S0, 16, N->Wl[7], 1, t);                /* dec0 */
    for (int64_t c = 0; c < L[0].cells; c++) z[c] = bf ? (double)((float)u[c] + (float)t[c]) : u[c] + t[c];
}

int dor_unet_forward(const int n[3], const float* w, const double* u, int bf, double* z, double* acts) {
    Net N;
    if (net_init(&N, n, w, bf)) return -1;
    net_forward(&N, u, bf, z);
    if (acts) {
        const Lev* L = N.lv;
        const double* src[7] = {N.S0, N.P1, N.S1, N.P2, N.S2, N.P3, N.E3};
        const int64_t len[7] = {L[0].cells * 16, L[1].cells * 16, L[1].cells * 32, L[2].cells * 32,
                                L[2].cells * 64, L[3].cells * 64, L[3].cells * 64};
        for (int a = 0; a < 7; a++) {
            memcpy(acts, src[a], sizeof(double) * len[a]);
            acts += len[a];
        }
    }
    net_free(&N);
    return 0;
}

int dor_unet_loss_grad(const int n[3], const float* w, const double* r, const double* e, int count, int bf,
                       double* loss, double* grad) {
    Net N;
    if (net_init(&N, n, w, bf)) return -1;
    const Lev* L = N.lv;
    const int64_t c0 = L[0].cells, c1 = L[1].cells, c2 = L[2].cells, c3 = L[3].cells;
    double* gW[8];
    int64_t off = 0;
    for (int l = 0; l < 8; l++) {
        gW[l] = grad ? grad + off : NULL;
        off += 27LL * kCin[l] * kCout[l];
    }
    if (grad) memset(grad, 0, sizeof(double) * off);
    double* z = (double*)malloc(sizeof(double) * c0);
    double* g = (double*)malloc(sizeof(double) * c0);
    double* dS0 = (double*)malloc(sizeof(double) * c0 * 16);
    double* dD1 = (double*)malloc(sizeof(double) * c1 * 16);
    double* dS1 = (double*)malloc(sizeof(double) * c1 * 32);
    double* dD2 = (double*)malloc(sizeof(double) * c2 * 32);
    double* dS2 = (double*)malloc(sizeof(double) * c2 * 64);
    double* dD3 = (double*)malloc(sizeof(double) * c3 * 64);
    double* dE3 = (double*)malloc(sizeof(double) * c3 * 64);
    double* dP = (double*)malloc(sizeof(double) * c1 * 64);
    const double scale = 1.0 / count;
    double ltot = 0.;
    for (int b = 0; b < count; b++) {
        const double* rb_ = r + (int64_t)b * c0;
        const double* eb = e + (int64_t)b * c0;
        net_forward(&N, rb_, bf, z);
        double en = 0., d2 = 0.;
        for (int64_t c = 0; c < c0; c++) en += eb[c] * eb[c];
        const double wgt = scale / (en > 1e-300 ? en : 1e-300);
        for (int64_t c = 0; c < c0; c++) {
            const double d = z[c] - eb[c];
            d2 += d * d;
            g[c] = 2. * wgt * d;
        }
        ltot += wgt * d2;
        if (!grad) continue;
        /* the weight and data gradients see the bf16 copy of g (embedded input) */
        for (int64_t c = 0; c < c0; c++) N.tmp[c] = bf ? rb(g[c]) : g[c];
        conv_w(&L[0], N.S0, 16, N.tmp, 1, 1.0, gW[7]);
        conv_t(&L[0], N.tmp, 1, N.Wl[7], 16, dS0);
        round_all(dS0, c0 * 16, bf);
        restrict2(&L[0], &L[1], dS0, 16, 1.0, dD1);
        round_all(dD1, c1 * 16, bf);
        conv_w(&L[1], N.S1, 32, dD1, 16, 1.0, gW[6]);
        conv_t(&L[1], dD1, 16, N.Wl[6], 32, dS1);
        round_all(dS1, c1 * 32, bf);
        restrict2(&L[1], &L[2], dS1, 32, 1.0, dD2);
        round_all(dD2, c2 * 32, bf);
        conv_w(&L[2], N.S2, 64, dD2, 32, 1.0, gW[5]);
        conv_t(&L[2], dD2, 32, N.Wl[5], 64, dS2);
        round_all(dS2, c2 * 64, bf);
        restrict2(&L[2], &L[3], dS2, 64, 1.0, dD3);
        round_all(dD3, c3 * 64, bf);
        conv_w(&L[3], N.E3, 64, dD3, 64, 1.0, gW[4]);
        conv_t(&L[3], dD3, 64, N.Wl[4], 64, dE3);
        round_all(dE3, c3 * 64, bf);
        conv_w(&L[3], N.P3, 64, dE3, 64, 1.0, gW[3]);
        conv_t(&L[3], dE3, 64, N.Wl[3], 64, dP);
        round_all(dP, c3 * 64, bf);
        prolong_add(&L[2], &L[3], dP, 64, 0.125, dS2, bf);
        conv_w(&L[2], N.P2, 32, dS2, 64, 1.0, gW[2]);
        conv_t(&L[2], dS2, 64, N.Wl[2], 32, dP);
        round_all(dP, c2 * 32, bf);
        prolong_add(&L[1], &L[2], dP, 32, 0.125, dS1, bf);
        conv_w(&L[1], N.P1, 16, dS1, 32, 1.0, gW[1]);
        conv_t(&L[1], dS1, 32, N.Wl[1], 16, dP);
        round_all(dP, c1 * 16, bf);
        prolong_add(&L[0], &L[1], dP, 16, 0.125, dS0, bf);
        conv_w(&L[0], N.x0, 1, dS0, 16, 1.0, gW[0]);
    }
    if (loss) *loss = ltot;
    free(z); free(g); free(dS0); free(dD1); free(dS1); free(dD2); free(dS2); free(dD3); free(dE3); free(dP);
    net_free(&N);
    return 0;
}
