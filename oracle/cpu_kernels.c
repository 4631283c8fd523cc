/*
 * CPU restatement of the reference's per-gate statevector kernels -- TEST
 * INFRASTRUCTURE ONLY (checker and timed CPU baseline; never on the product path).
 *
 * One full pass over the state per gate, as the reference's kernels do:
 *   1q gate on pair (i0, i0 + 2^q)             qgpusim_cuda/src/kernels.cu:10-50
 *   2q gate, matrix index b_q0 + 2*b_q1         kernels.cu:56-137
 *   out-of-place bit-permutation scatter        kernels.cu:165-185
 * Complex numbers are interleaved (re, im); matrices are row-major.
 * Parallelised with OpenMP over the pair / quadruple index.
 */
#include <stdint.h>
#include <string.h>
#include <omp.h>

#define DEFINE_KERNELS(SUF, R)                                                             \
void qo_apply_1q_##SUF(R *psi, int n, int q, const R *U) {                               \
    const int64_t half = (int64_t)1 << (n - 1);                                            \
    const int64_t stride = (int64_t)1 << q;                                                \
    const R u0r = U[0], u0i = U[1], u1r = U[2], u1i = U[3];                                \
    const R u2r = U[4], u2i = U[5], u3r = U[6], u3i = U[7];                                \
    _Pragma("omp parallel for schedule(static)")                                           \
    for (int64_t k = 0; k < half; ++k) {                                                   \
        int64_t i0 = ((k >> q) << (q + 1)) | (k & (stride - 1));                           \
        int64_t i1 = i0 + stride;                                                          \
        R ar = psi[2 * i0], ai = psi[2 * i0 + 1], br = psi[2 * i1], bi = psi[2 * i1 + 1];   \
        psi[2 * i0] = u0r * ar - u0i * ai + u1r * br - u1i * bi;                           \
        psi[2 * i0 + 1] = u0r * ai + u0i * ar + u1r * bi + u1i * br;                       \
        psi[2 * i1] = u2r * ar - u2i * ai + u3r * br - u3i * bi;                           \
        psi[2 * i1 + 1] = u2r * ai + u2i * ar + u3r * bi + u3i * br;                       \
    }                                                                                      \
}                                                                                          \
void qo_apply_2q_##SUF(R *psi, int n, int q0, int q1, const R *U) {                       \
    const int lo = q0 < q1 ? q0 : q1, hi = q0 < q1 ? q1 : q0;                              \
    const int64_t quarter = (int64_t)1 << (n - 2);                                         \
    const int64_t mlo = (int64_t)1 << lo, mhi = (int64_t)1 << hi;                          \
    /* offsets of matrix index b_q0 + 2*b_q1 */                                            \
    const int64_t m0 = (int64_t)1 << q0, m1 = (int64_t)1 << q1;                            \
    const int64_t off[4] = {0, m0, m1, m0 | m1};                                           \
    _Pragma("omp parallel for schedule(static)")                                           \
    for (int64_t k = 0; k < quarter; ++k) {                                                \
        int64_t base = k & (mlo - 1);                                                      \
        base |= ((k >> lo) & ((mhi >> (lo + 1)) - 1)) << (lo + 1);                         \
        base |= (k >> (hi - 1)) << (hi + 1);                                               \
        R vr[4], vi[4];                                                                    \
        for (int c = 0; c < 4; ++c) { vr[c] = psi[2 * (base + off[c])];                    \
                                      vi[c] = psi[2 * (base + off[c]) + 1]; }              \
        for (int r = 0; r < 4; ++r) {                                                      \
            R sr = 0, si = 0;                                                              \
            for (int c = 0; c < 4; ++c) {                                                  \
                R ur = U[2 * (4 * r + c)], ui = U[2 * (4 * r + c) + 1];                     \
                sr += ur * vr[c] - ui * vi[c];                                             \
                si += ur * vi[c] + ui * vr[c];                                             \
            }                                                                              \
            psi[2 * (base + off[r])] = sr;                                                 \
            psi[2 * (base + off[r]) + 1] = si;                                             \
        }                                                                                  \
    }                                                                                      \
}                                                                                          \
void qo_permute_scatter_##SUF(const R *in, R *out, int n, const int *map_old_to_new) {     \
    const int64_t dim = (int64_t)1 << n;                                                   \
    _Pragma("omp parallel for schedule(static)")                                           \
    for (int64_t i = 0; i < dim; ++i) {                                                    \
        int64_t j = 0;                                                                     \
        for (int p = 0; p < n; ++p) j |= ((i >> p) & 1) << map_old_to_new[p];              \
        out[2 * j] = in[2 * i];                                                            \
        out[2 * j + 1] = in[2 * i + 1];                                                    \
    }                                                                                      \
}                                                                                          \
/* Runs ops in order: kind 1 = 1q (q0, U[0..7]), kind 2 = 2q (q0, q1, U[0..31]).         \
   Matrices are packed at 32 reals per op. */                                              \
void qo_run_ops_##SUF(R *psi, int n, int nops, const int *kind, const int *q0,             \
                      const int *q1, const R *Us) {                                        \
    for (int k = 0; k < nops; ++k) {                                                       \
        if (kind[k] == 1) qo_apply_1q_##SUF(psi, n, q0[k], Us + 32 * (int64_t)k);          \
        else qo_apply_2q_##SUF(psi, n, q0[k], q1[k], Us + 32 * (int64_t)k);                 \
    }                                                                                      \
}

DEFINE_KERNELS(c64, float)
DEFINE_KERNELS(c128, double)

int qo_max_threads(void) { return omp_get_max_threads(); }
void qo_set_threads(int t) { if (t > 0) omp_set_num_threads(t); }
