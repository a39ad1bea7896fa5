// Krylov drivers on the device (FP64): preconditioned CG and restarted,
// right-preconditioned GMRES(m).  They stand in for Krylov.jl's CG/GMRES,
// which the reference reaches through LinearSolve.jl (Pl = P,
// test/test_preconditioners.jl:65,93) and which calls ldiv!(y, P, x) once per
// iteration.
//
// PCG keeps every scalar on the device.  One iteration (SpMV fused with p.q,
// alpha fused with the x/r update and r.r, convergence test, M^-1 r, r.z,
// beta fused with the p update) is captured once as a CUDA graph and replayed
// in batches; the
// convergence test freezes x and r on the iteration that meets
// ||r|| <= rtol ||b||, so replaying past convergence changes nothing and the
// reported iteration count is the first one that met the test.
//
// Arithmetic.  Dot products and norms are compensated (Dot2) sums and every
// vector update is separately rounded (no FMA contraction), the same
// arithmetic the CPU restatement uses, so with the bitwise-identical SpMV and
// preconditioners the device iterates reproduce the restatement's.
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"
#include "reduce.cuh"
#include "spmv.cuh"

namespace {

constexpr int kT = 256;

struct PcgScalars {
    double bb, rr, rz, pq, alpha, beta, rtol;
    double eps, rnorm;   // Krylov.jl test: sqrt(r.z) <= eps = atol + rtol sqrt(r0.z0)
    int done, it, conv_it, pad;
};

inline int grid_elems(int64_t n) {
    const int64_t b = (n + kT - 1) / kT;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)hs::num_sms() * 8));
}

// Streaming kernels work on tiles of kU x kT elements: each thread issues the
// loads of its kU elements before using any of them, so every thread keeps kU
// elements per stream in flight.  blockDim.x must be kT.
constexpr int kU = 4;
constexpr int64_t kTile = (int64_t)kU * kT;

// Blocks for a tiled streaming kernel: at most 4 per SM (and kRedMaxBlocks),
// with the tiles spread evenly over them.
inline int tile_blocks(int64_t n) {
    const int64_t tiles = std::max<int64_t>(1, (n + kTile - 1) / kTile);
    const int64_t maxb = std::min<int64_t>((int64_t)hs::num_sms() * 4, hsdev::kRedMaxBlocks);
    const int64_t per = (tiles + maxb - 1) / maxb;
    return (int)((tiles + per - 1) / per);
}

__global__ void copy_kernel(int64_t n, const double* __restrict__ a, double* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

__global__ void zero_kernel(int64_t n, double* __restrict__ a) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = 0.0;
}

using hsdev::DD;

__device__ __forceinline__ void store_dd(double* partials, DD v) {
    v = hsdev::block_dd(v);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = v.s;
        partials[2 * blockIdx.x + 1] = v.c;
    }
}

// compensated partial sums of a.b: partials[2*block], partials[2*block+1]
__global__ void __launch_bounds__(kT) dot_kernel(int64_t n, const double* __restrict__ a,
                                                 const double* __restrict__ b, double* __restrict__ partials) {
    DD v{0.0, 0.0};
    for (int64_t base = blockIdx.x * kTile + threadIdx.x; base < n; base += (int64_t)gridDim.x * kTile) {
        double xa[kU], xb[kU];
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const int64_t i = base + k * kT;
            if (i < n) {
                xa[k] = a[i];
                xb[k] = b[i];
            }
        }
#pragma unroll
        for (int k = 0; k < kU; ++k)
            if (base + k * kT < n) hsdev::dd_add_prod(v, xa[k], xb[k]);
    }
    store_dd(partials, v);
}

// Sum of compensated partials; valid on thread 0.
__device__ __forceinline__ double sum_partials(const double* __restrict__ partials, int nb) {
    DD v{0.0, 0.0};
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v = hsdev::dd_add(v, DD{partials[2 * i], partials[2 * i + 1]});
    return hsdev::dd_value(hsdev::block_dd(v));
}

// The same sum (thread 0's value) on every thread of the block.
__device__ __forceinline__ double sum_partials_all(const double* __restrict__ partials, int nb) {
    DD v{0.0, 0.0};
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v = hsdev::dd_add(v, DD{partials[2 * i], partials[2 * i + 1]});
    return hsdev::dd_value(hsdev::block_dd_all(v));
}

// kjl: Krylov.jl's stopping test (sqrt(r.z) <= atol + rtol sqrt(r0.z0)),
// else ||r|| <= rtol ||b||.
__global__ void pcg_init_scalars(const double* __restrict__ partials_bb, const double* __restrict__ partials_rz,
                                 int nb, PcgScalars* s, double rtol, double atol, int kjl) {
    const double bb = sum_partials(partials_bb, nb);
    __syncthreads();
    const double rz = sum_partials(partials_rz, nb);
    if (threadIdx.x == 0) {
        s->bb = bb;
        s->rr = bb;
        s->rz = rz;
        s->rtol = rtol;
        s->rnorm = sqrt(rz);
        s->eps = __dadd_rn(atol, __dmul_rn(rtol, s->rnorm));
        s->done = kjl ? (rz == 0.0 || s->rnorm <= s->eps) : (bb == 0.0);
        s->it = 0;
        s->conv_it = s->done ? 0 : -1;
    }
}

// Krylov.jl's test after z = M^-1 r: rNorm = sqrt(r.z) <= eps (or rNorm + 1
// <= 1); a non-positive p.q (no curvature) stops without convergence.
__global__ void kjl_check(const double* __restrict__ partials, int nb, PcgScalars* s) {
    const double rz = sum_partials(partials, nb);
    if (threadIdx.x == 0 && !s->done) {
        s->it += 1;
        if (!(s->pq > 0.0)) {
            s->done = 2;
            return;
        }
        const double rn = sqrt(rz);
        s->rnorm = rn;
        if (rn <= s->eps || __dadd_rn(rn, 1.0) <= 1.0) {
            s->done = 1;
            s->conv_it = s->it;
        }
    }
}

// q = A p (storage-order rows, bitwise mul!) and compensated partials of p.q.
// A warp owns 32 rows at a time (warp CSR-stream), warps stride over the matrix.
// q = A p with the p.q partials over the matrix's 32-row slices (spmv.cuh):
// the same row sums bit for bit as the CSR kernel below, with each lane's
// row entries loaded eight at a time.  Each warp takes every (grid x 8)-th
// slice; the next slice's bounds are loaded one slice ahead.
__global__ void __launch_bounds__(kT, 4) pcg_spmv_dot_sliced(int32_t n, const int64_t* __restrict__ soff,
                                                         const int32_t* __restrict__ scol,
                                                         const double* __restrict__ sval,
                                                         const double* __restrict__ p, double* __restrict__ q,
                                                         const PcgScalars* __restrict__ s,
                                                         double* __restrict__ partials) {
    DD part{0.0, 0.0};
    const int64_t nsl = ((int64_t)n + 31) / 32;
    const int64_t stride = (int64_t)gridDim.x * (kT / 32);
    int64_t sl = (int64_t)blockIdx.x * (kT / 32) + (threadIdx.x >> 5);
    int64_t o0 = sl < nsl ? soff[sl] : 0, o1 = sl < nsl ? soff[sl + 1] : 0;
    if (!s->done) {
        auto fp = [&](int32_t j) { return __ldg(p + j); };
        for (; sl < nsl; sl += stride) {
            const int64_t nx = sl + stride;
            const int64_t n0 = nx < nsl ? soff[nx] : 0, n1 = nx < nsl ? soff[nx + 1] : 0;
            const double acc = hsdev::slice_row_sum(o0, o1, scol, sval, fp);
            const int64_t r = sl * 32 + (threadIdx.x & 31);
            if (r < n) {
                q[r] = acc;
                hsdev::dd_add_prod(part, p[r], acc);
            }
            o0 = n0;
            o1 = n1;
        }
    }
    store_dd(partials, part);
}

// alpha = r.z / p.q (every block sums the partials itself, in the same order,
// so every block holds the same alpha); x += alpha p; r -= alpha q; partials
// of r.r.  Skipped (r.r only) once converged.
__global__ void __launch_bounds__(kT) pcg_update(int64_t n, PcgScalars* __restrict__ s, const double* __restrict__ ppq,
                                                 int npq, const double* __restrict__ prz, int nrz,
                                                 const double* __restrict__ p, const double* __restrict__ q,
                                                 double* __restrict__ x, double* __restrict__ r,
                                                 double* __restrict__ partials) {
    const bool done = s->done;
    const double rz = sum_partials_all(prz, nrz);
    const double pq = sum_partials_all(ppq, npq);
    const double alpha = __ddiv_rn(rz, pq);
    if (blockIdx.x == 0 && threadIdx.x == 0 && !done) {
        s->rz = rz;
        s->pq = pq;
        s->alpha = alpha;
    }
    DD v{0.0, 0.0};
    for (int64_t base = blockIdx.x * kTile + threadIdx.x; base < n; base += (int64_t)gridDim.x * kTile) {
        double xv[kU], pv[kU], rv[kU], qv[kU];
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const int64_t i = base + k * kT;
            if (i < n) {
                rv[k] = r[i];
                if (!done) {
                    xv[k] = x[i];
                    pv[k] = p[i];
                    qv[k] = q[i];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const int64_t i = base + k * kT;
            if (i < n) {
                if (!done) {
                    x[i] = __dadd_rn(xv[k], __dmul_rn(alpha, pv[k]));
                    rv[k] = __dsub_rn(rv[k], __dmul_rn(alpha, qv[k]));
                    r[i] = rv[k];
                }
                hsdev::dd_add_prod(v, rv[k], rv[k]);
            }
        }
    }
    store_dd(partials, v);
}

__global__ void pcg_check(const double* __restrict__ partials, int nb, PcgScalars* s) {
    const double rr = sum_partials(partials, nb);
    if (threadIdx.x == 0) {
        if (!s->done) {
            s->it += 1;
            s->rr = rr;
            if (sqrt(rr) <= __dmul_rn(s->rtol, sqrt(s->bb))) {
                s->done = 1;
                s->conv_it = s->it;
            }
        }
    }
}

// beta = r.z_new / r.z (every block sums the r.z partials itself); p = z + beta p.
__global__ void __launch_bounds__(kT) pcg_p(int64_t n, const PcgScalars* __restrict__ s,
                                            const double* __restrict__ prz, int nrz, const double* __restrict__ z,
                                            double* __restrict__ p) {
    if (s->done) return;
    const double beta = __ddiv_rn(sum_partials_all(prz, nrz), s->rz);
    for (int64_t base = blockIdx.x * kTile + threadIdx.x; base < n; base += (int64_t)gridDim.x * kTile) {
        double zv[kU], pv[kU];
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const int64_t i = base + k * kT;
            if (i < n) {
                zv[k] = z[i];
                pv[k] = p[i];
            }
        }
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const int64_t i = base + k * kT;
            if (i < n) p[i] = __dadd_rn(zv[k], __dmul_rn(beta, pv[k]));
        }
    }
}

int prec_apply(int type, void* prec, const double* r, double* z, int64_t n, cudaStream_t st) {
    if (type == HS_PREC_L1GS) return hs_l1gs_apply(static_cast<hs_l1gs*>(prec), r, z, HS_F64, st);
    if (type == HS_PREC_CHEB) return hs::cheb_apply(static_cast<hs_cheb*>(prec), r, z, HS_F64, st);
    copy_kernel<<<grid_elems(n), kT, 0, st>>>(n, r, z);
    HS_LAUNCH_CHECK("copy_kernel");
    return HS_OK;
}

struct DevBuf {
    std::vector<void*> ptrs;
    ~DevBuf() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    int alloc(T** p, size_t bytes) {
        cudaError_t e = cudaMalloc((void**)p, bytes ? bytes : 8);
        if (e != cudaSuccess) return hs::cuda_error(e, "cudaMalloc (krylov)");
        ptrs.push_back(*p);
        return HS_OK;
    }
};

// *out = sum of compensated partials (sqrt of it when sqrt_out).
__global__ void finalize_dd_kernel(const double* __restrict__ partials, int nb, double* __restrict__ out,
                                   int sqrt_out) {
    const double v = sum_partials(partials, nb);
    if (threadIdx.x == 0) *out = sqrt_out ? sqrt(v) : v;
}

double true_relres(hs_matrix* A, const double* b, const double* x, double* work, double* partials, double* scal,
                   int64_t n, cudaStream_t st, double bnorm) {
    copy_kernel<<<grid_elems(n), kT, 0, st>>>(n, b, work);
    hs::matrix_spmv(A, x, work, -1.0, 1.0, st);
    const int nb = hsdev::red_blocks(n);
    dot_kernel<<<nb, kT, 0, st>>>(n, work, work, partials);
    finalize_dd_kernel<<<1, kT, 0, st>>>(partials, nb, scal, 1);
    hs::count_launch(3);
    double v = 0;
    cudaMemcpyAsync(&v, scal, 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return bnorm > 0 ? v / bnorm : 0.0;
}

// ---- GMRES helpers (every operation separately rounded, as in the oracle) --
// partials[2*(i*nb + block)] = compensated V_i . w  for i < jc
__global__ void mdot_kernel(int64_t n, const double* __restrict__ V, int64_t ldv, int jc, const double* __restrict__ w,
                            double* __restrict__ partials, int nb) {
    for (int i = 0; i < jc; ++i) {
        const double* Vi = V + (size_t)i * ldv;
        DD v{0.0, 0.0};
        for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
            hsdev::dd_add_prod(v, Vi[r], w[r]);
        v = hsdev::block_dd(v);
        if (threadIdx.x == 0) {
            partials[2 * ((size_t)i * nb + blockIdx.x)] = v.s;
            partials[2 * ((size_t)i * nb + blockIdx.x) + 1] = v.c;
        }
        __syncthreads();
    }
}

// hcol[i] = sum of partials row i; H[i][j] += hcol[i]   (grid = jc blocks)
__global__ void mdot_finalize(const double* __restrict__ partials, int nb, double* __restrict__ hcol,
                              double* __restrict__ H, int m, int j) {
    const int i = blockIdx.x;
    const double v = sum_partials(partials + 2 * (size_t)i * nb, nb);
    if (threadIdx.x == 0) {
        hcol[i] = v;
        H[(size_t)i * m + j] = __dadd_rn(H[(size_t)i * m + j], v);
    }
}

// w -= sum_i hcol[i] V_i, in order i = 0..jc-1
__global__ void gs_update(int64_t n, const double* __restrict__ V, int64_t ldv, int jc, const double* __restrict__ hcol,
                          double* __restrict__ w) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double s = w[r];
        for (int i = 0; i < jc; ++i) s = __dsub_rn(s, __dmul_rn(hcol[i], V[(size_t)i * ldv + r]));
        w[r] = s;
    }
}

// H[j+1][j] = ||w||, Givens update; flag = converged/breakdown
__global__ void arnoldi_close(const double* __restrict__ partials, int nb, double* __restrict__ H, int m, int j,
                              double* __restrict__ cs, double* __restrict__ sn, double* __restrict__ g,
                              double* __restrict__ hn_out, int* __restrict__ flag, double tol) {
    const double ss = sum_partials(partials, nb);
    if (threadIdx.x != 0) return;
    const double hn = sqrt(ss);
    *hn_out = hn;
    H[(size_t)(j + 1) * m + j] = hn;
    for (int i = 0; i < j; ++i) {
        const double a0 = H[(size_t)i * m + j], a1 = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = __dadd_rn(__dmul_rn(cs[i], a0), __dmul_rn(sn[i], a1));
        H[(size_t)(i + 1) * m + j] = __dadd_rn(__dmul_rn(-sn[i], a0), __dmul_rn(cs[i], a1));
    }
    const double a0 = H[(size_t)j * m + j], a1 = H[(size_t)(j + 1) * m + j];
    const double den = sqrt(__dadd_rn(__dmul_rn(a0, a0), __dmul_rn(a1, a1)));
    const double c = den == 0.0 ? 1.0 : __ddiv_rn(a0, den), s = den == 0.0 ? 0.0 : __ddiv_rn(a1, den);
    cs[j] = c;
    sn[j] = s;
    H[(size_t)j * m + j] = __dadd_rn(__dmul_rn(c, a0), __dmul_rn(s, a1));
    H[(size_t)(j + 1) * m + j] = 0.0;
    g[j + 1] = __dmul_rn(-s, g[j]);
    g[j] = __dmul_rn(c, g[j]);
    *flag = (fabs(g[j + 1]) <= tol || hn == 0.0) ? 1 : 0;
}

__global__ void scale_from(int64_t n, const double* __restrict__ w, const double* __restrict__ hn, double* __restrict__ out) {
    const double h = *hn;
    if (h == 0.0) return;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        out[r] = __ddiv_rn(w[r], h);
}

__global__ void back_solve(const double* __restrict__ H, int m, int jend, const double* __restrict__ g, double* __restrict__ y) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = jend - 1; i >= 0; --i) {
        double s = g[i];
        for (int t = i + 1; t < jend; ++t) s = __dsub_rn(s, __dmul_rn(H[(size_t)i * m + t], y[t]));
        y[i] = __ddiv_rn(s, H[(size_t)i * m + i]);
    }
}

// t = sum_i y_i V_i, in order i = 0..jc-1 from 0
__global__ void combine(int64_t n, const double* __restrict__ V, int64_t ldv, int jc, const double* __restrict__ y,
                        double* __restrict__ t) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < jc; ++i) s = __dadd_rn(s, __dmul_rn(y[i], V[(size_t)i * ldv + r]));
        t[r] = s;
    }
}

__global__ void add_to(int64_t n, const double* __restrict__ u, double* __restrict__ x) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        x[r] = __dadd_rn(x[r], u[r]);
}

__global__ void set_g(double* g, int m, double beta) {
    for (int i = threadIdx.x; i <= m; i += blockDim.x) g[i] = (i == 0) ? beta : 0.0;
}

// ---- Krylov.jl GMRES helpers ---------------------------------------------
// q -= h V_i with h = V_i.q summed from the partials by every block in the
// same order; block 0 records h as R[i][k].
__global__ void __launch_bounds__(kT) mgs_axpy(int64_t n, const double* __restrict__ partials, int nb,
                                               const double* __restrict__ Vi, double* __restrict__ q,
                                               double* __restrict__ Rik) {
    const double h = sum_partials_all(partials, nb);
    if (blockIdx.x == 0 && threadIdx.x == 0) *Rik = h;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        q[r] = __dsub_rn(q[r], __dmul_rn(h, Vi[r]));
}

__device__ __forceinline__ double sgn(double a) { return a < 0.0 ? -1.0 : 1.0; }

// Symmetric Givens reflection [c s; s -c] [a; b] = [rho; 0] (Krylov.jl's
// sym_givens; Golub & Van Loan / Bindel, Demmel & Kahan).
__device__ void sym_givens(double a, double b, double* c, double* s, double* rho) {
    if (b == 0.0) {
        *c = (a == 0.0) ? 1.0 : sgn(a);
        *s = 0.0;
        *rho = fabs(a);
    } else if (a == 0.0) {
        *c = 0.0;
        *s = sgn(b);
        *rho = fabs(b);
    } else if (fabs(b) > fabs(a)) {
        const double t = __ddiv_rn(a, b);
        *s = __ddiv_rn(sgn(b), sqrt(__dadd_rn(1.0, __dmul_rn(t, t))));
        *c = __dmul_rn(*s, t);
        *rho = __ddiv_rn(b, *s);
    } else {
        const double t = __ddiv_rn(b, a);
        *c = __ddiv_rn(sgn(a), sqrt(__dadd_rn(1.0, __dmul_rn(t, t))));
        *s = __dmul_rn(*c, t);
        *rho = __ddiv_rn(a, *c);
    }
}

// Closes inner iteration k: Hbis = ||q||, previous reflections applied to
// column k of R, a new one from (R_kk, Hbis), zeta = s_k z_k, z_k = c_k z_k,
// z_{k+1} = zeta; scal[0] = Hbis, scal[1] = |zeta|; flag = solved | 2*breakdown.
__global__ void kjl_arnoldi_close(const double* __restrict__ partials, int nb, double* __restrict__ R, int m, int k,
                                  double* __restrict__ c, double* __restrict__ sv, double* __restrict__ z,
                                  double* __restrict__ scal, int* __restrict__ flag, double eps, double btol) {
    const double qq = sum_partials(partials, nb);
    if (threadIdx.x != 0) return;
    const double hbis = sqrt(qq);
    for (int i = 0; i < k; ++i) {
        const double ri = R[(size_t)i * m + k], ri1 = R[(size_t)(i + 1) * m + k];
        const double tmp = __dadd_rn(__dmul_rn(c[i], ri), __dmul_rn(sv[i], ri1));
        R[(size_t)(i + 1) * m + k] = __dsub_rn(__dmul_rn(sv[i], ri), __dmul_rn(c[i], ri1));
        R[(size_t)i * m + k] = tmp;
    }
    double ck, sk, rho;
    sym_givens(R[(size_t)k * m + k], hbis, &ck, &sk, &rho);
    c[k] = ck;
    sv[k] = sk;
    R[(size_t)k * m + k] = rho;
    const double zeta = __dmul_rn(sk, z[k]);
    z[k] = __dmul_rn(ck, z[k]);
    z[k + 1] = zeta;
    const double rn = fabs(zeta);
    scal[0] = hbis;
    scal[1] = rn;
    const bool solved = rn <= eps || __dadd_rn(rn, 1.0) <= 1.0;
    *flag = (solved ? 1 : 0) | (hbis <= btol ? 2 : 0);
}

// y = R \ z over the first kk columns: y_i = (z_i - sum_{j>i, from the last}
// R_ij y_j) / R_ii, or 0 where |R_ii| <= btol.
__global__ void kjl_back_solve(const double* __restrict__ R, int m, int kk, const double* __restrict__ z,
                               double* __restrict__ y, double btol) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = kk - 1; i >= 0; --i) {
        double yi = z[i];
        for (int j = kk - 1; j > i; --j) yi = __dsub_rn(yi, __dmul_rn(R[(size_t)i * m + j], y[j]));
        const double rii = R[(size_t)i * m + i];
        y[i] = fabs(rii) <= btol ? 0.0 : __ddiv_rn(yi, rii);
    }
}

// w = b - w
__global__ void rsub_kernel(int64_t n, const double* __restrict__ b, double* __restrict__ w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        w[i] = __dsub_rn(b[i], w[i]);
}

// One PCG driver, two stopping tests: kjl = false, ||r|| <= rtol ||b||
// checked after the x/r update (hs_pcg_solve); kjl = true, Krylov.jl's cg
// test checked after z = M^-1 r (hs_cg_krylovjl).
int pcg_impl(hs_matrix* A, int32_t prec_type, void* prec, const double* b, double* x, double atol, double rtol,
             int32_t maxit, void* stream, hs_solve_info* info, bool kjl) {
    if (!A || !b || !x || !info) return hs::set_error(HS_ERR_ARG, "hs_pcg_solve: NULL argument");
    if (prec_type != HS_PREC_NONE && !prec) return hs::set_error(HS_ERR_ARG, "preconditioner handle is NULL");
    if (kjl && maxit == 0) maxit = 2 * hs::matrix_n(A);   // Krylov.jl's itmax = 0: 2n
    if (maxit < 1) return hs::set_error(HS_ERR_ARG, "maxit must be positive");
    if (!(rtol >= 0.0) || !(atol >= 0.0)) return hs::set_error(HS_ERR_ARG, "tolerances must be non-negative");
    // The solve runs on a private non-blocking stream (graph capture is not
    // allowed on the legacy default stream), ordered after and before the
    // caller's stream by events.
    cudaStream_t caller = static_cast<cudaStream_t>(stream);
    // Stream, event and workspace are kept per calling thread and per device
    // (a stream belongs to the device it was made on): repeated solves (a
    // Krylov loop inside a time stepper, a served stream) pay no
    // cudaMalloc/cudaFree, and no device synchronisation of cudaFree, per
    // solve.  The workspace grows on demand.
    int dev = 0;
    HS_CUDA(cudaGetDevice(&dev));
    constexpr int kMaxDevices = 64;
    if (dev < 0 || dev >= kMaxDevices) return hs::set_error(HS_ERR_UNSUPPORTED, "device ordinal %d above 63", dev);
    static thread_local struct Ctx {
        cudaStream_t own = nullptr;
        cudaEvent_t join = nullptr;
        int64_t cap = 0;
        double* base = nullptr;
    } ctxs[kMaxDevices];
    Ctx& ws = ctxs[dev];
    if (!ws.own) {
        HS_CUDA(cudaStreamCreateWithFlags(&ws.own, cudaStreamNonBlocking));
        HS_CUDA(cudaEventCreateWithFlags(&ws.join, cudaEventDisableTiming));
    }
    cudaStream_t own = ws.own;
    cudaEvent_t join = ws.join;
    HS_CUDA(cudaEventRecord(join, caller));
    HS_CUDA(cudaStreamWaitEvent(own, join, 0));
    cudaStream_t st = own;
    struct Rejoin {
        cudaStream_t a, b;
        cudaEvent_t e;
        ~Rejoin() {
            cudaEventRecord(e, a);
            cudaStreamWaitEvent(b, e, 0);
        }
    } rejoin{own, caller, join};
    const int64_t n = hs::matrix_n(A);
    const int64_t need = 4 * n + 6 * hsdev::kRedMaxBlocks + 2 + (int64_t)(sizeof(PcgScalars) / 8 + 1);
    if (ws.cap < need) {
        if (ws.base) {
            HS_CUDA(cudaStreamSynchronize(own));   // earlier solves on this device may still read it
            cudaFree(ws.base);
        }
        ws.base = nullptr;
        ws.cap = 0;
        HS_CUDA(cudaMalloc(&ws.base, sizeof(double) * need));
        ws.cap = need;
    }
    double* r = ws.base;
    double* z = r + n;
    double* p = z + n;
    double* q = p + n;
    double* pa = q + n;
    double* pb = pa + 2 * hsdev::kRedMaxBlocks;
    double* pc = pb + 2 * hsdev::kRedMaxBlocks;
    double* scal = pc + 2 * hsdev::kRedMaxBlocks;
    PcgScalars* s = reinterpret_cast<PcgScalars*>(scal + 2);
    int rc;
    const int ge = grid_elems(n), nb = tile_blocks(n);
    // Timing events and the iteration graph are released on every return path.
    struct Owned {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        ~Owned() {
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } own_res;
    HS_CUDA(cudaEventCreate(&own_res.e0));
    HS_CUDA(cudaEventCreate(&own_res.e1));
    cudaEvent_t e0 = own_res.e0, e1 = own_res.e1;
    cudaEventRecord(e0, st);
    // x = 0, r = b, z = M^-1 r, p = z
    zero_kernel<<<ge, kT, 0, st>>>(n, x);
    copy_kernel<<<ge, kT, 0, st>>>(n, b, r);
    hs::count_launch(2);
    if ((rc = prec_apply(prec_type, prec, r, z, n, st))) return rc;
    copy_kernel<<<ge, kT, 0, st>>>(n, z, p);
    dot_kernel<<<nb, kT, 0, st>>>(n, b, b, pa);
    dot_kernel<<<nb, kT, 0, st>>>(n, r, z, pb);
    pcg_init_scalars<<<1, kT, 0, st>>>(pa, pb, nb, s, rtol, atol, kjl ? 1 : 0);
    hs::count_launch(4);
    HS_LAUNCH_CHECK("pcg init");

    // One iteration as a graph: q = A p with the p.q partials (pa); alpha,
    // x/r update and r.r partials (pc); convergence test; z = M^-1 r; r.z
    // partials (pb); beta and p update.
    const int32_t *Arp = nullptr, *Aci = nullptr;
    const void* Av = nullptr;
    int Adt = 0;
    hs::matrix_arrays(A, &Arp, &Aci, &Av, &Adt);
    const int64_t* Asoff = nullptr;
    const int32_t* Ascol = nullptr;
    const void* Asv = nullptr;
    if (Adt == HS_F64 && (rc = hs::matrix_slices(A, st, &Asoff, &Ascol, &Asv))) return rc;
    const double* Asval = static_cast<const double*>(Asv);
    const int nq = (int)std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, (int64_t)hsdev::kRedMaxBlocks));
    auto iteration = [&](cudaStream_t cs) -> int {
        int r2;
        int npq = nb;
        if (Adt == HS_F64) {
            pcg_spmv_dot_sliced<<<nq, kT, 0, cs>>>((int32_t)n, Asoff, Ascol, Asval, p, q, s, pa);
            npq = nq;
        } else {
            if ((r2 = hs::matrix_spmv(A, p, q, 1.0, 0.0, cs))) return r2;
            dot_kernel<<<nb, kT, 0, cs>>>(n, p, q, pa);
        }
        pcg_update<<<nb, kT, 0, cs>>>(n, s, pa, npq, pb, nb, p, q, x, r, pc);
        if (!kjl) pcg_check<<<1, kT, 0, cs>>>(pc, nb, s);
        hs::count_launch(kjl ? 2 : 3);   // spmv (+dot), update, check
        if ((r2 = prec_apply(prec_type, prec, r, z, n, cs))) return r2;
        dot_kernel<<<nb, kT, 0, cs>>>(n, r, z, pb);
        if (kjl) kjl_check<<<1, kT, 0, cs>>>(pb, nb, s);
        pcg_p<<<nb, kT, 0, cs>>>(n, s, pb, nb, z, p);
        hs::count_launch(kjl ? 2 : 1);   // dot (+ check); the check below counts pcg_p
        HS_LAUNCH_CHECK("pcg iteration");
        return HS_OK;
    };
    // warm launch outside capture (sets kernel attributes), then capture
    cudaGraph_t& graph = own_res.graph;
    cudaGraphExec_t& exec = own_res.exec;
    bool use_graph = true;
    if ((rc = iteration(st))) return rc;
    int launches_per_iter = 0;
    {
        const int64_t before = hs_kernel_launches();
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            use_graph = false;
            cudaGetLastError();
        } else {
            rc = iteration(st);
            cudaError_t ce = cudaStreamEndCapture(st, &graph);
            if (rc || ce != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
                use_graph = false;
                cudaGetLastError();
            }
        }
        launches_per_iter = (int)(hs_kernel_launches() - before);
        hs::count_launch(-launches_per_iter);  // counted per replay below
    }
    PcgScalars hsc{};
    int iters_run = 1;
    const int batch = 8;
    while (true) {
        HS_CUDA(cudaMemcpyAsync(&hsc, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
        HS_CUDA(cudaStreamSynchronize(st));
        if (hsc.done || iters_run >= maxit) break;
        const int todo = std::min(batch, maxit - iters_run);
        for (int k = 0; k < todo; ++k) {
            if (use_graph) {
                HS_CUDA(cudaGraphLaunch(exec, st));
                hs::count_launch(launches_per_iter);
            } else if ((rc = iteration(st))) {
                return rc;
            }
        }
        iters_run += todo;
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double bnorm = std::sqrt(hsc.bb);
    const bool conv = hsc.done == 1;
    info->iterations = conv ? hsc.conv_it : hsc.it;
    info->converged = conv ? 1 : 0;
    info->ms = ms;
    info->relres = true_relres(A, b, x, q, pa, scal, n, st, bnorm);
    info->rnorm = kjl ? hsc.rnorm : std::sqrt(hsc.rr);
    HS_CUDA(cudaGetLastError());
    if (hsc.done == 2) return hs::set_error(HS_ERR_NOT_CONVERGED, "CG stopped: p.q <= 0 (no positive curvature)");
    if (!conv) return hs::set_error(HS_ERR_NOT_CONVERGED, "PCG did not converge in %d iterations", maxit);
    return HS_OK;
}

}  // namespace

extern "C" {

int hs_pcg_solve(hs_matrix* A, int32_t prec_type, void* prec, const double* b, double* x, double rtol, int32_t maxit,
                 void* stream, hs_solve_info* info) {
    return pcg_impl(A, prec_type, prec, b, x, 0.0, rtol, maxit, stream, info, false);
}

int hs_cg_krylovjl(hs_matrix* A, int32_t prec_type, void* prec, const double* b, double* x, double atol, double rtol,
                   int32_t itmax, void* stream, hs_solve_info* info) {
    return pcg_impl(A, prec_type, prec, b, x, atol, rtol, itmax, stream, info, true);
}

// Krylov.jl's gmres with restart and a left preconditioner (LinearSolve's
// KrylovJL_GMRES with Pl = P, restart length `memory`): the residual
// estimate |zeta| of ||M^-1 (b - A x)|| is tested against
// atol + rtol ||M^-1 b|| after every inner iteration.
int hs_gmres_krylovjl(hs_matrix* A, int32_t prec_type, void* prec, int32_t memory, const double* b, double* x,
                      double atol, double rtol, int32_t itmax, void* stream, hs_solve_info* info) {
    if (!A || !b || !x || !info) return hs::set_error(HS_ERR_ARG, "hs_gmres_krylovjl: NULL argument");
    if (prec_type != HS_PREC_NONE && !prec) return hs::set_error(HS_ERR_ARG, "preconditioner handle is NULL");
    if (memory < 1 || memory > 1024) return hs::set_error(HS_ERR_ARG, "memory (restart length) must be in 1..1024");
    if (itmax < 0 || !(rtol >= 0.0) || !(atol >= 0.0)) return hs::set_error(HS_ERR_ARG, "bad itmax or tolerances");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = hs::matrix_n(A);
    if (itmax == 0) itmax = (int32_t)std::min<int64_t>(2 * n, INT32_MAX);
    const int m = memory;
    const double btol = std::pow(2.220446049250313e-16, 0.75);
    DevBuf buf;
    double *V, *w, *q, *partials, *R, *c, *sv, *z, *y, *scal;
    int* flag;
    int rc;
    if ((rc = buf.alloc(&V, 8 * (size_t)n * (m + 1))) || (rc = buf.alloc(&w, 8 * n)) || (rc = buf.alloc(&q, 8 * n)) ||
        (rc = buf.alloc(&partials, 16 * (size_t)hsdev::kRedMaxBlocks)) ||
        (rc = buf.alloc(&R, 8 * (size_t)(m + 1) * m)) || (rc = buf.alloc(&c, 8 * m)) || (rc = buf.alloc(&sv, 8 * m)) ||
        (rc = buf.alloc(&z, 8 * (m + 1))) || (rc = buf.alloc(&y, 8 * m)) || (rc = buf.alloc(&scal, 16)) ||
        (rc = buf.alloc(&flag, sizeof(int))))
        return rc;
    const int ge = grid_elems(n), nb = hsdev::red_blocks(n);
    struct Events {   // released on every return path
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } evs;
    HS_CUDA(cudaEventCreate(&evs.e0));
    HS_CUDA(cudaEventCreate(&evs.e1));
    cudaEventRecord(evs.e0, st);
    auto norm_to = [&](const double* a, double* out) {   // *out = ||a|| on the device
        dot_kernel<<<nb, kT, 0, st>>>(n, a, a, partials);
        finalize_dd_kernel<<<1, kT, 0, st>>>(partials, nb, out, 1);
        hs::count_launch(2);
    };
    auto read = [&](const double* d) -> double {
        double v = 0;
        cudaMemcpyAsync(&v, d, 8, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        return v;
    };
    zero_kernel<<<ge, kT, 0, st>>>(n, x);
    hs::count_launch();
    // r0 = M \ b in V_0's storage; beta0 = ||r0||
    if ((rc = prec_apply(prec_type, prec, b, V, n, st))) return rc;
    norm_to(V, scal + 1);
    double beta = read(scal + 1);
    double rn = beta;
    const double eps = atol + rtol * rn;
    int32_t iter = 0, npass = 0;
    bool solved = rn <= eps, breakdown = false;
    while (!(solved || iter >= itmax || breakdown)) {
        HS_CUDA(cudaMemsetAsync(R, 0, 8 * (size_t)(m + 1) * m, st));
        HS_CUDA(cudaMemsetAsync(z, 0, 8 * (size_t)(m + 1), st));
        if (npass >= 1) {   // r0 = M \ (b - A x)
            if ((rc = hs::matrix_spmv(A, x, w, 1.0, 0.0, st))) return rc;
            rsub_kernel<<<ge, kT, 0, st>>>(n, b, w);
            hs::count_launch();
            if ((rc = prec_apply(prec_type, prec, w, V, n, st))) return rc;
            norm_to(V, scal + 1);
            beta = read(scal + 1);
        }
        HS_CUDA(cudaMemcpyAsync(z, &beta, 8, cudaMemcpyHostToDevice, st));
        scale_from<<<ge, kT, 0, st>>>(n, V, scal + 1, V);   // V_0 = r0 / beta
        hs::count_launch();
        ++npass;
        int k = 0;
        while (true) {
            const double* Vk = V + (size_t)k * n;
            if ((rc = hs::matrix_spmv(A, Vk, w, 1.0, 0.0, st))) return rc;
            if ((rc = prec_apply(prec_type, prec, w, q, n, st))) return rc;
            for (int i = 0; i <= k; ++i) {   // modified Gram-Schmidt
                const double* Vi = V + (size_t)i * n;
                dot_kernel<<<nb, kT, 0, st>>>(n, Vi, q, partials);
                mgs_axpy<<<ge, kT, 0, st>>>(n, partials, nb, Vi, q, R + (size_t)i * m + k);
                hs::count_launch(2);
            }
            dot_kernel<<<nb, kT, 0, st>>>(n, q, q, partials);
            kjl_arnoldi_close<<<1, kT, 0, st>>>(partials, nb, R, m, k, c, sv, z, scal, flag, eps, btol);
            hs::count_launch(2);
            int hflag = 0;
            HS_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
            HS_CUDA(cudaStreamSynchronize(st));
            ++iter;
            ++k;
            solved = (hflag & 1) != 0;
            breakdown = (hflag & 2) != 0;
            if (solved || breakdown || k >= m || iter >= itmax) break;
            scale_from<<<ge, kT, 0, st>>>(n, q, scal, V + (size_t)k * n);   // V_k = q / Hbis
            hs::count_launch();
        }
        rn = read(scal + 1);
        kjl_back_solve<<<1, 32, 0, st>>>(R, m, k, z, y, btol);
        combine<<<ge, kT, 0, st>>>(n, V, n, k, y, w);
        add_to<<<ge, kT, 0, st>>>(n, w, x);
        hs::count_launch(3);
    }
    cudaEventRecord(evs.e1, st);
    cudaEventSynchronize(evs.e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, evs.e0, evs.e1);
    // true relative residual of x
    copy_kernel<<<ge, kT, 0, st>>>(n, b, w);
    hs::count_launch();
    if ((rc = hs::matrix_spmv(A, x, w, -1.0, 1.0, st))) return rc;
    norm_to(w, scal);
    norm_to(b, scal + 1);
    const double rr = read(scal), bn = read(scal + 1);
    HS_CUDA(cudaGetLastError());
    info->iterations = iter;
    info->converged = solved ? 1 : 0;
    info->relres = bn > 0 ? rr / bn : 0.0;
    info->rnorm = rn;
    info->ms = ms;
    if (!solved) return hs::set_error(HS_ERR_NOT_CONVERGED, "GMRES did not converge in %d iterations", itmax);
    return HS_OK;
}

int hs_gmres_solve(hs_matrix* A, int32_t prec_type, void* prec, int32_t restart, const double* b, double* x, double rtol,
                   int32_t maxit, void* stream, hs_solve_info* info) {
    if (!A || !b || !x || !info) return hs::set_error(HS_ERR_ARG, "hs_gmres_solve: NULL argument");
    if (prec_type != HS_PREC_NONE && !prec) return hs::set_error(HS_ERR_ARG, "preconditioner handle is NULL");
    if (restart < 1 || restart > 256 || maxit < 1) return hs::set_error(HS_ERR_ARG, "bad restart/maxit");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = hs::matrix_n(A);
    const int m = restart;
    DevBuf buf;
    double *V, *u, *w, *r, *partials, *H, *cs, *sn, *g, *y, *hcol, *scal;
    int* flag;
    int rc;
    if ((rc = buf.alloc(&V, 8 * (size_t)n * (m + 1))) || (rc = buf.alloc(&u, 8 * n)) || (rc = buf.alloc(&w, 8 * n)) ||
        (rc = buf.alloc(&r, 8 * n)) || (rc = buf.alloc(&partials, 16 * (size_t)hsdev::kRedMaxBlocks * (m + 1))) ||
        (rc = buf.alloc(&H, 8 * (size_t)(m + 1) * m)) || (rc = buf.alloc(&cs, 8 * m)) || (rc = buf.alloc(&sn, 8 * m)) ||
        (rc = buf.alloc(&g, 8 * (m + 1))) || (rc = buf.alloc(&y, 8 * m)) || (rc = buf.alloc(&hcol, 8 * (m + 1))) ||
        (rc = buf.alloc(&scal, 16)) || (rc = buf.alloc(&flag, sizeof(int))))
        return rc;
    const int ge = grid_elems(n), nb = hsdev::red_blocks(n);
    struct Events {   // released on every return path
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } evs;
    HS_CUDA(cudaEventCreate(&evs.e0));
    HS_CUDA(cudaEventCreate(&evs.e1));
    cudaEvent_t e0 = evs.e0, e1 = evs.e1;
    cudaEventRecord(e0, st);
    auto norm = [&](const double* a) -> double {
        dot_kernel<<<nb, kT, 0, st>>>(n, a, a, partials);
        finalize_dd_kernel<<<1, kT, 0, st>>>(partials, nb, scal, 1);
        hs::count_launch(2);
        double v = 0;
        cudaMemcpyAsync(&v, scal, 8, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        return v;
    };
    zero_kernel<<<ge, kT, 0, st>>>(n, x);
    copy_kernel<<<ge, kT, 0, st>>>(n, b, r);
    hs::count_launch(2);
    const double bnorm = norm(b);
    double beta = bnorm;
    int total = 0;
    bool conv = bnorm == 0.0;
    const double tol = rtol * bnorm;
    while (!conv && total < maxit) {
        // V0 = r / beta
        {
            double* vb = scal + 1;
            HS_CUDA(cudaMemcpyAsync(vb, &beta, 8, cudaMemcpyHostToDevice, st));
            scale_from<<<ge, kT, 0, st>>>(n, r, vb, V);
            hs::count_launch();
        }
        HS_CUDA(cudaMemsetAsync(H, 0, 8 * (size_t)(m + 1) * m, st));
        set_g<<<1, 64, 0, st>>>(g, m, beta);
        hs::count_launch();
        int jend = 0;
        for (int j = 0; j < m; ++j) {
            double* Vj = V + (size_t)j * n;
            if ((rc = prec_apply(prec_type, prec, Vj, u, n, st))) return rc;
            if ((rc = hs::matrix_spmv(A, u, w, 1.0, 0.0, st))) return rc;
            for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
                mdot_kernel<<<nb, kT, 0, st>>>(n, V, n, j + 1, w, partials, nb);
                mdot_finalize<<<j + 1, kT, 0, st>>>(partials, nb, hcol, H, m, j);
                gs_update<<<ge, kT, 0, st>>>(n, V, n, j + 1, hcol, w);
                hs::count_launch(3);
            }
            dot_kernel<<<nb, kT, 0, st>>>(n, w, w, partials);
            arnoldi_close<<<1, kT, 0, st>>>(partials, nb, H, m, j, cs, sn, g, scal, flag, tol);
            scale_from<<<ge, kT, 0, st>>>(n, w, scal, V + (size_t)(j + 1) * n);
            hs::count_launch(3);
            int hflag = 0;
            HS_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
            HS_CUDA(cudaStreamSynchronize(st));
            ++total;
            jend = j + 1;
            if (hflag || total >= maxit) break;
        }
        back_solve<<<1, 32, 0, st>>>(H, m, jend, g, y);
        combine<<<ge, kT, 0, st>>>(n, V, n, jend, y, w);
        hs::count_launch(2);
        if ((rc = prec_apply(prec_type, prec, w, u, n, st))) return rc;
        add_to<<<ge, kT, 0, st>>>(n, u, x);
        copy_kernel<<<ge, kT, 0, st>>>(n, b, r);
        hs::count_launch(2);
        if ((rc = hs::matrix_spmv(A, x, r, -1.0, 1.0, st))) return rc;
        beta = norm(r);
        if (beta <= tol) conv = true;
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    HS_CUDA(cudaGetLastError());
    info->iterations = total;
    info->converged = conv ? 1 : 0;
    info->relres = bnorm > 0 ? beta / bnorm : 0.0;
    info->rnorm = beta;
    info->ms = ms;
    if (!conv) return hs::set_error(HS_ERR_NOT_CONVERGED, "GMRES did not converge in %d iterations", maxit);
    return HS_OK;
}

}  // extern "C"
