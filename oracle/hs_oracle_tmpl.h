/*
 * CPU oracle for the HybridSmoothers.jl preconditioner-apply path — TEST
 * INFRASTRUCTURE ONLY.  Nothing in the product library links or calls this
 * code; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it, as the checker.
 *
 * This header is included twice by hs_oracle.c, once with REAL=double and once
 * with REAL=float, so every routine exists as *_f64 and *_f32.  Each routine
 * restates the Julia reference (HybridSmoothers.jl v0.1.4); the citation in
 * front of each one is `file:line` inside that project.
 *
 * Arithmetic contract (what makes bit-exact parity possible):
 *   - Julia evaluates `acc += a*b` as round(acc + round(a*b)); it never fuses
 *     into an FMA without @fastmath/@muladd.  This file is compiled with
 *     -ffp-contract=off so C does the same.
 *   - Summation order is the reference's: ascending column within a row for
 *     every accumulation (packed, view, CSR, CSC binary search, l1 row sums,
 *     SpMV).
 *   - Indices are 0-based here; the reference is 1-based.  Every offset
 *     formula below is the reference formula shifted by one.
 *
 * Matrices are "row-wise" triples (rp, ci, v): row pointer (n+1), column index
 * and value arrays.  The reference reads row i from
 *   - CSR:            the CSR row,
 *   - symmetric CSC:  column i of the CSC (isSymA=true takes column i as row i),
 *   - non-symmetric CSC: the true row, which it gathers by binary search over
 *     columns (literal restatements of that path are the *_csc_nonsym
 *     functions below).
 */

#define CAT2_(a, b) a##b
#define CAT2(a, b) CAT2_(a, b)
#define F(name) CAT2(name, SFX)

/* ------------------------------------------------------------------------ */
/* Partition geometry: l1_gauss_seidel.jl:946-958 (_makecache).              */
/* ------------------------------------------------------------------------ */
static inline void F(part_range)(int32_t n, int32_t ps, int64_t k, int32_t* s, int32_t* e)
{
    int64_t start = k * (int64_t)ps;
    int64_t end = start + ps - 1;
    if (end > n - 1) end = n - 1;
    *s = (int32_t)start;
    *e = (int32_t)end;
}

/* Packed buffer length S: l1_gauss_seidel.jl:699-701. */
int64_t F(hso_packed_size)(int32_t n, int32_t ps)
{
    int64_t nparts = ((int64_t)n + ps - 1) / ps;
    int64_t lps = (int64_t)n - (nparts - 1) * ps;
    return ((int64_t)ps * (ps - 1) * (nparts - 1)) / 2 + (lps * (lps - 1)) / 2;
}

/* ------------------------------------------------------------------------ */
/* D_Dl1 for one row from a row-wise scan.                                   */
/*   scan: l1_gauss_seidel.jl:1101-1129 (_diag_offpart_rowwise)              */
/*   rule: l1_gauss_seidel.jl:1017-1022 (eta test, dl1/2)                    */
/* ------------------------------------------------------------------------ */
static inline REAL F(dl1_row)(const int32_t* rp, const int32_t* ci, const REAL* v,
                              int32_t i, int32_t s, int32_t e, REAL eta)
{
    REAL b = (REAL)0, d = (REAL)0;
    for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
        int32_t j = ci[p];
        REAL val = v[p];
        if (j == i)
            b = val;
        else if (j < s || j > e)
            d += ABS(val);
    }
    REAL dl1star = (b >= eta * d) ? (REAL)0 : d / (REAL)2;
    return b + dl1star;
}

/*
 * D_Dl1 for every row, iterating partitions the way DiagonalPartsIterator does
 * (l1_gauss_seidel.jl:913-944): work item g in [0, nchunks*chunksize) handles
 * partitions g, g+stride, ...  Results do not depend on nchunks/chunksize; the
 * iteration is mirrored so the invariance tests exercise it.
 * Kernel restated: _compute_D_Dl1_kernel! l1_gauss_seidel.jl:993-1024.
 */
void F(hso_dl1_rowwise)(int32_t n, const int32_t* rp, const int32_t* ci, const REAL* v,
                        int32_t ps, double eta_in, int32_t nchunks, int32_t chunksize, REAL* D)
{
    const REAL eta = (REAL)eta_in; /* convert(Tf, η), l1_gauss_seidel.jl:969 */
    const int64_t nparts = ((int64_t)n + ps - 1) / ps;
    const int64_t stride = (int64_t)nchunks * chunksize;
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < stride; ++g) {
        for (int64_t k = g; k < nparts; k += stride) {
            int32_t s, e;
            F(part_range)(n, ps, k, &s, &e);
            for (int32_t i = s; i <= e; ++i) D[i] = F(dl1_row)(rp, ci, v, i, s, e, eta);
        }
    }
}

/*
 * Literal restatement of the non-symmetric CSC D_Dl1 scan
 * (_diag_offpart(::NonSymmetricMatrix, ::CSCFormat, ...), l1_gauss_seidel.jl:1135-1216):
 * for every row, loop over ALL columns and binary-search the row inside the
 * below-/above-diagonal segment given by DiagonalIndices.  O(N^2 log); only
 * for small cross-checks of hso_dl1_rowwise on the transposed matrix.
 */
void F(hso_dl1_csc_nonsym_literal)(int32_t n, const int32_t* colptr, const int32_t* rowval,
                                   const REAL* nzval, const int32_t* diag, int32_t ps,
                                   double eta_in, REAL* D)
{
    const REAL eta = (REAL)eta_in;
    const int64_t nparts = ((int64_t)n + ps - 1) / ps;
    for (int64_t k = 0; k < nparts; ++k) {
        int32_t s, e;
        F(part_range)(n, ps, k, &s, &e);
        for (int32_t idx = s; idx <= e; ++idx) {
            REAL b = nzval[diag[idx]];
            REAL d = (REAL)0;
            for (int32_t col = 0; col < idx; ++col) { /* :1156-1183 */
                if (!(col < s || col > e)) continue;
                int32_t p_lo = diag[col] + 1, p_hi = colptr[col + 1] - 1;
                if (p_lo > p_hi) continue;
                if (rowval[p_lo] <= idx && rowval[p_hi] >= idx) {
                    int32_t left = p_lo, right = p_hi;
                    while (left <= right) {
                        int32_t mid = (left + right) >> 1;
                        int32_t row = rowval[mid];
                        if (row < idx) left = mid + 1;
                        else if (row > idx) right = mid - 1;
                        else { d += ABS(nzval[mid]); break; }
                    }
                }
            }
            for (int32_t col = idx + 1; col < n; ++col) { /* :1186-1213 */
                if (!(col < s || col > e)) continue;
                int32_t p_lo = colptr[col], p_hi = diag[col] - 1;
                if (p_lo > p_hi) continue;
                if (rowval[p_lo] <= idx && rowval[p_hi] >= idx) {
                    int32_t left = p_lo, right = p_hi;
                    while (left <= right) {
                        int32_t mid = (left + right) >> 1;
                        int32_t row = rowval[mid];
                        if (row < idx) left = mid + 1;
                        else if (row > idx) right = mid - 1;
                        else { d += ABS(nzval[mid]); break; }
                    }
                }
            }
            REAL dl1star = (b >= eta * d) ? (REAL)0 : d / (REAL)2;
            D[idx] = b + dl1star;
        }
    }
}

/*
 * DiagonalIndices(A) for CSC, l1_gauss_seidel.jl:422-436: position of A[c,c]
 * inside rowval (0-based here).  Returns -1 on success, else the 0-based
 * column whose diagonal is missing or zero (the reference throws
 * SingularException(col) with the 1-based column).
 */
int32_t F(hso_diag_indices)(int32_t n, const int32_t* colptr, const int32_t* rowval,
                            const REAL* nzval, int32_t* diag)
{
    for (int32_t col = 0; col < n; ++col) {
        int32_t r1 = colptr[col], r2 = colptr[col + 1] - 1;
        /* searchsortedfirst(rowval, col, r1, r2) */
        int32_t lo = r1, hi = r2 + 1;
        while (lo < hi) {
            int32_t mid = lo + ((hi - lo) >> 1);
            if (rowval[mid] < col) lo = mid + 1; else hi = mid;
        }
        r1 = lo;
        if (r1 > r2 || rowval[r1] != col || nzval[r1] == (REAL)0) return col;
        diag[col] = r1;
    }
    return -1;
}

/* ------------------------------------------------------------------------ */
/* Packing, reference layout.                                               */
/*   lower: block k at k*ps(ps-1)/2, row li at li(li-1)/2, column lj.        */
/*   upper: block k at k*ps(ps-1)/2, row li at li*aps - li(li+1)/2 (aps =    */
/*          actual partsize of this block), element j at (j - i - 1).        */
/* ------------------------------------------------------------------------ */

/* _pack_strict_lower_rowwise!, l1_gauss_seidel.jl:1248-1277 */
static void F(pack_lower_rowwise_part)(const int32_t* rp, const int32_t* ci, const REAL* v,
                                       int32_t s, int32_t e, int32_t ps, int64_t k, REAL* SL)
{
    const int64_t block_offset = k * (((int64_t)ps * (ps - 1)) / 2);
    for (int32_t i = s; i <= e; ++i) {
        int64_t li = i - s;
        int64_t row_offset = (li * (li - 1)) / 2;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            int32_t j = ci[p];
            if (j >= s && j < i) SL[block_offset + row_offset + (j - s)] = v[p];
        }
    }
}

/* _pack_strict_upper_rowwise!, l1_gauss_seidel.jl:1380-1413 */
static void F(pack_upper_rowwise_part)(const int32_t* rp, const int32_t* ci, const REAL* v,
                                       int32_t s, int32_t e, int32_t ps, int64_t k, REAL* SU)
{
    const int64_t block_offset = k * (((int64_t)ps * (ps - 1)) / 2);
    const int64_t aps = (int64_t)e - s + 1;
    for (int32_t i = s; i <= e; ++i) {
        int64_t li = i - s;
        int64_t row_start = li * aps - (li * (li + 1)) / 2;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            int32_t j = ci[p];
            if (j > i && j <= e) SU[block_offset + row_start + (j - i) - 1] = v[p];
        }
    }
}

/*
 * _precompute_and_pack_kernel!, l1_gauss_seidel.jl:1028-1066: D_Dl1 plus the
 * strict lower and/or upper packed triangles (SL/SU must be zero-filled by the
 * caller, as the reference allocates them with zeros(), :702, :749, :796-797).
 */
void F(hso_l1gs_setup_rowwise)(int32_t n, const int32_t* rp, const int32_t* ci, const REAL* v,
                               int32_t ps, double eta, int32_t nchunks, int32_t chunksize,
                               REAL* D, REAL* SL, REAL* SU)
{
    const REAL eta_c = (REAL)eta;
    const int64_t nparts = ((int64_t)n + ps - 1) / ps;
    const int64_t stride = (int64_t)nchunks * chunksize;
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < stride; ++g) {
        for (int64_t k = g; k < nparts; k += stride) {
            int32_t s, e;
            F(part_range)(n, ps, k, &s, &e);
            for (int32_t i = s; i <= e; ++i) D[i] = F(dl1_row)(rp, ci, v, i, s, e, eta_c);
            if (SL) F(pack_lower_rowwise_part)(rp, ci, v, s, e, ps, k, SL);
            if (SU) F(pack_upper_rowwise_part)(rp, ci, v, s, e, ps, k, SU);
        }
    }
}

/* Non-symmetric CSC packing, lower: l1_gauss_seidel.jl:1279-1324 (literal). */
void F(hso_pack_lower_csc_nonsym)(int32_t n, const int32_t* colptr, const int32_t* rowval,
                                  const REAL* nzval, int32_t ps, REAL* SL)
{
    const int64_t nparts = ((int64_t)n + ps - 1) / ps;
    for (int64_t k = 0; k < nparts; ++k) {
        int32_t s, e;
        F(part_range)(n, ps, k, &s, &e);
        const int64_t block_offset = k * (((int64_t)ps * (ps - 1)) / 2);
        for (int32_t col = s; col <= e - 1; ++col) {
            int64_t lj = col - s;
            int32_t p = colptr[col], col_end = colptr[col + 1];
            while (p < col_end && rowval[p] <= col) ++p;
            while (p < col_end) {
                int32_t i = rowval[p];
                if (i > e) break;
                int64_t li = i - s;
                SL[block_offset + (li * (li - 1)) / 2 + lj] = nzval[p];
                ++p;
            }
        }
    }
}

/* Non-symmetric CSC packing, upper: l1_gauss_seidel.jl:1415-1469 (literal). */
void F(hso_pack_upper_csc_nonsym)(int32_t n, const int32_t* colptr, const int32_t* rowval,
                                  const REAL* nzval, int32_t ps, REAL* SU)
{
    const int64_t nparts = ((int64_t)n + ps - 1) / ps;
    for (int64_t k = 0; k < nparts; ++k) {
        int32_t s, e;
        F(part_range)(n, ps, k, &s, &e);
        const int64_t block_offset = k * (((int64_t)ps * (ps - 1)) / 2);
        const int64_t aps = (int64_t)e - s + 1;
        for (int32_t col = s + 1; col <= e; ++col) {
            int64_t lj = col - s;
            for (int32_t p = colptr[col]; p < colptr[col + 1]; ++p) {
                int32_t i = rowval[p];
                if (i < col) {
                    if (i < s) continue;
                    int64_t li = i - s;
                    int64_t row_start = li * aps - (li * (li + 1)) / 2;
                    SU[block_offset + row_start + (lj - li) - 1] = nzval[p];
                } else {
                    break;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Sweeps.                                                                  */
/* ------------------------------------------------------------------------ */

/* Packed lower accumulation, l1_gauss_seidel.jl:1547-1562. */
static inline REAL F(acc_packed_lower)(const REAL* SL, const REAL* y, int32_t i, int64_t k,
                                       int32_t ps, int32_t s)
{
    const int64_t block_offset = k * (((int64_t)ps * (ps - 1)) / 2);
    const int64_t li = i - s;
    const int64_t row_offset = (li * (li - 1)) / 2;
    REAL acc = (REAL)0;
    for (int64_t lj = 0; lj < li; ++lj) acc += SL[block_offset + row_offset + lj] * y[s + lj];
    return acc;
}

/* Packed upper accumulation, l1_gauss_seidel.jl:1564-1585. */
static inline REAL F(acc_packed_upper)(const REAL* SU, const REAL* y, int32_t i, int64_t k,
                                       int32_t ps, int32_t s, int32_t e)
{
    const int64_t block_offset = k * (((int64_t)ps * (ps - 1)) / 2);
    const int64_t aps = (int64_t)e - s + 1;
    const int64_t li = i - s;
    const int64_t row_start = li * aps - (li * (li + 1)) / 2;
    const int64_t num_upper = aps - 1 - li;
    REAL acc = (REAL)0;
    for (int64_t o = 1; o <= num_upper; ++o) {
        int64_t gj = i + o;
        if (gj > e) break;
        acc += SU[block_offset + row_start + o - 1] * y[gj];
    }
    return acc;
}

/* Row-wise view accumulations, l1_gauss_seidel.jl:1588-1597 and :1700-1709. */
static inline REAL F(acc_view_lower)(const int32_t* rp, const int32_t* ci, const REAL* v,
                                     const REAL* y, int32_t i, int32_t s)
{
    REAL acc = (REAL)0;
    for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
        int32_t j = ci[p];
        if (s <= j && j < i) acc += v[p] * y[j];
    }
    return acc;
}
static inline REAL F(acc_view_upper)(const int32_t* rp, const int32_t* ci, const REAL* v,
                                     const REAL* y, int32_t i, int32_t e)
{
    REAL acc = (REAL)0;
    for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
        int32_t j = ci[p];
        if (i < j && j <= e) acc += v[p] * y[j];
    }
    return acc;
}

/* Non-symmetric CSC binary-search accumulation, l1_gauss_seidel.jl:1616-1650,
 * lower range :1663-1664, upper range :1694-1695. */
static inline REAL F(acc_csc_binsearch)(const int32_t* colptr, const int32_t* rowval,
                                        const REAL* nzval, const int32_t* diag, const REAL* y,
                                        int32_t i, int32_t c0, int32_t c1, int lower)
{
    REAL acc = (REAL)0;
    for (int32_t col = c0; col <= c1; ++col) {
        int32_t p_lo, p_hi;
        if (lower) { p_lo = diag[col] + 1; p_hi = colptr[col + 1] - 1; }
        else       { p_lo = colptr[col];   p_hi = diag[col] - 1; }
        if (p_lo <= p_hi && rowval[p_lo] <= i && rowval[p_hi] >= i) {
            int32_t left = p_lo, right = p_hi;
            while (left <= right) {
                int32_t mid = (left + right) >> 1;
                if (rowval[mid] < i) left = mid + 1;
                else if (rowval[mid] > i) right = mid - 1;
                else { acc += nzval[mid] * y[col]; break; }
            }
        }
    }
    return acc;
}

/*
 * One directional sweep over every partition, in place on y
 * (_apply_sweep_kernel!, l1_gauss_seidel.jl:1068-1095; rows ascending for a
 * lower cache, descending for an upper cache, sweep_range :450-451).
 *   kind 0: packed (SL or SU), 1: row-wise view, 2: non-symmetric CSC view.
 */
static void F(sweep_dir)(int32_t n, int32_t ps, int lower, int kind,
                         const REAL* buf, const int32_t* rp, const int32_t* ci, const REAL* v,
                         const int32_t* diag, const REAL* D, REAL* y,
                         int32_t nchunks, int32_t chunksize)
{
    const int64_t nparts = ((int64_t)n + ps - 1) / ps;
    const int64_t stride = (int64_t)nchunks * chunksize;
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < stride; ++g) {
        for (int64_t k = g; k < nparts; k += stride) {
            int32_t s, e;
            F(part_range)(n, ps, k, &s, &e);
            if (lower) {
                for (int32_t i = s; i <= e; ++i) {
                    REAL acc;
                    if (kind == 0) acc = F(acc_packed_lower)(buf, y, i, k, ps, s);
                    else if (kind == 1) acc = F(acc_view_lower)(rp, ci, v, y, i, s);
                    else acc = F(acc_csc_binsearch)(rp, ci, v, diag, y, i, s, (i - 1 < e ? i - 1 : e), 1);
                    y[i] = (y[i] - acc) / D[i];
                }
            } else {
                for (int32_t i = e; i >= s; --i) {
                    REAL acc;
                    if (kind == 0) acc = F(acc_packed_upper)(buf, y, i, k, ps, s, e);
                    else if (kind == 1) acc = F(acc_view_upper)(rp, ci, v, y, i, e);
                    else acc = F(acc_csc_binsearch)(rp, ci, v, diag, y, i, i + 1, e, 0);
                    y[i] = (y[i] - acc) / D[i];
                }
            }
        }
    }
}

/*
 * ldiv!(y, P, x): y .= x, then the sweep plan (l1_gauss_seidel.jl:386-396,
 * :854-877 for Forward/Backward, :880-906 for Symmetric: forward with the
 * lower cache, y .= D_Dl1 .* y, backward with the upper cache).
 *   sweep: 0 forward, 1 backward, 2 symmetric.
 *   kind:  0 packed (SL, SU in the reference layout), 1 row-wise view
 *          (symmetric CSC or CSR), 2 non-symmetric CSC view (rp/ci/v are
 *          colptr/rowval/nzval and diag is DiagonalIndices).
 */
void F(hso_l1gs_apply)(int32_t n, int32_t ps, int32_t sweep, int32_t kind,
                       const REAL* SL, const REAL* SU,
                       const int32_t* rp, const int32_t* ci, const REAL* v, const int32_t* diag,
                       const REAL* D, const REAL* x, REAL* y, int32_t nchunks, int32_t chunksize)
{
    if (y != x) memcpy(y, x, sizeof(REAL) * (size_t)n);
    if (sweep == 0 || sweep == 2)
        F(sweep_dir)(n, ps, 1, kind, SL, rp, ci, v, diag, D, y, nchunks, chunksize);
    if (sweep == 2) {
        for (int32_t i = 0; i < n; ++i) y[i] = D[i] * y[i]; /* :897 */
    }
    if (sweep == 1 || sweep == 2)
        F(sweep_dir)(n, ps, 0, kind, SU, rp, ci, v, diag, D, y, nchunks, chunksize);
}

/* ------------------------------------------------------------------------ */
/* Chebyshev smoothers (chebyshev.jl).                                      */
/* ------------------------------------------------------------------------ */

/* _l1_rowsum, chebyshev.jl:27-36: l1[row] += |a| over columns ascending. */
void F(hso_l1_rowsum_csc)(int32_t n, const int32_t* colptr, const int32_t* rowval,
                          const REAL* nzval, REAL* l1)
{
    for (int32_t i = 0; i < n; ++i) l1[i] = (REAL)0;
    for (int32_t col = 0; col < n; ++col)
        for (int32_t p = colptr[col]; p < colptr[col + 1]; ++p) l1[rowval[p]] += ABS(nzval[p]);
}

/*
 * y = A*x for CSR (three-argument mul!).  The reference calls
 * SparseMatricesCSR.jl (compat 0.6, not vendored) at chebyshev.jl:47,165,287,305;
 * restated from that package's published algorithm: y[row] starts at zero and
 * accumulates nzval*x[col] over the row's entries in storage order.
 */
void F(hso_spmv)(int32_t n, const int32_t* rp, const int32_t* ci, const REAL* v,
                 const REAL* x, REAL* y)
{
#pragma omp parallel for schedule(static)
    for (int32_t row = 0; row < n; ++row) {
        REAL acc = (REAL)0;
        for (int32_t p = rp[row]; p < rp[row + 1]; ++p) acc += v[p] * x[ci[p]];
        y[row] = acc;
    }
}

/*
 * r = r - A*z (five-argument mul!(r, A, z, -1, 1), chebyshev.jl:179): with
 * beta == 1 the package leaves r in place and adds (nzval*z[col])*alpha term by
 * term into r[row]; (a*z)*(-1) is exactly -(a*z).
 */
void F(hso_spmv_sub)(int32_t n, const int32_t* rp, const int32_t* ci, const REAL* v,
                     const REAL* z, REAL* r)
{
#pragma omp parallel for schedule(static)
    for (int32_t row = 0; row < n; ++row) {
        REAL acc = r[row];
        for (int32_t p = rp[row]; p < rp[row + 1]; ++p) acc = acc + (v[p] * z[ci[p]]) * (REAL)(-1);
        r[row] = acc;
    }
}

/*
 * Power iteration for rho(M^-1 A), chebyshev.jl:40-54.  norm(w) in the
 * reference is LinearAlgebra.norm (BLAS nrm2 for n >= 32), whose summation
 * order is library-specific; here it is sqrt of the ascending sum of squares.
 * rho therefore agrees with the reference to rounding, not bitwise.
 */
double F(hso_power_rho)(int32_t n, const int32_t* rp, const int32_t* ci, const REAL* v,
                        const REAL* l1inv, int32_t iters, REAL* work_v, REAL* work_w)
{
    REAL init = (REAL)1 / SQRT((REAL)n);
    for (int32_t i = 0; i < n; ++i) work_v[i] = init;
    REAL rho = (REAL)1;
    for (int32_t it = 0; it < iters; ++it) {
        F(hso_spmv)(n, rp, ci, v, work_v, work_w);
        for (int32_t i = 0; i < n; ++i) work_w[i] *= l1inv[i];
        double ss = 0.0;
        for (int32_t i = 0; i < n; ++i) ss += (double)work_w[i] * (double)work_w[i];
        rho = (REAL)sqrt(ss);
        if (rho == (REAL)0) break;
        for (int32_t i = 0; i < n; ++i) work_v[i] = work_w[i] / rho;
    }
    return (double)rho;
}

/*
 * ChebyshevFourth smooth!, chebyshev.jl:158-183.  rho, l1inv as built by
 * _build_smoother (:141-156).  r and z are the smoother's work vectors.
 * Coefficients are computed in double and rounded to REAL, as the reference
 * does with T((2k-3)/(2k+1)) and T((8k-4)/((2k+1)*rho)) (:173-174).
 */
void F(hso_cheb4_smooth)(int32_t n, const int32_t* rp, const int32_t* ci, const REAL* v,
                         const REAL* l1inv, double rho, int32_t degree,
                         REAL* x, const REAL* b, REAL* r, REAL* z)
{
    F(hso_spmv)(n, rp, ci, v, x, r);                      /* :165 */
    for (int32_t i = 0; i < n; ++i) r[i] = b[i] - r[i];  /* :167, kernel :61-64 */
    for (int32_t i = 0; i < n; ++i) z[i] = (REAL)0;      /* :170 */
    for (int32_t k = 1; k <= degree; ++k) {
        REAL ak = (REAL)((double)(2 * k - 3) / (double)(2 * k + 1));
        REAL bk = (REAL)((double)(8 * k - 4) / ((double)(2 * k + 1) * rho));
        for (int32_t i = 0; i < n; ++i) {                /* kernel :132-139 */
            REAL zi = ak * z[i] + (bk * l1inv[i]) * r[i];
            z[i] = zi;
            x[i] += zi;
        }
        F(hso_spmv_sub)(n, rp, ci, v, z, r);              /* :179 */
    }
}

/* _cheb1_astar, chebyshev.jl:81-89 (bisection on x = sqrt(a*), 60 steps). */
double F(hso_cheb1_astar)(int32_t k)
{
    double lo = 1e-10, hi = 1.0 - 1e-10;
    for (int it = 0; it < 60; ++it) {
        double mid = (lo + hi) / 2;
        double phi = 8.0 * k * pow(1 - mid * mid, 2 * k) +
                     mid * (pow(1 - mid, 4 * k) - pow(1 + mid, 4 * k));
        if (phi > 0) lo = mid; else hi = mid;
    }
    double m = (lo + hi) / 2;
    return m * m;
}

/*
 * ChebyshevFirst smooth!, chebyshev.jl:278-322, with kernels :237-256 and
 * :67-70.  The scalar recurrence (a*, 1/rho, rho_k, c1, c2) runs in double, as
 * the reference does for Float64 data (:283-284, :296, :311-314); each scalar
 * is rounded to REAL where it meets a vector, so the f64 variant is the
 * reference's Float64 arithmetic and the f32 variant is "FP64 scalars, FP32
 * vectors".
 */
void F(hso_cheb1_smooth)(int32_t n, const int32_t* rp, const int32_t* ci, const REAL* v,
                         const REAL* l1inv, double rho, double astar, int32_t degree,
                         REAL* x, const REAL* b, REAL* r, REAL* z, REAL* tmp)
{
    const double a = astar;
    const REAL inv_rho = (REAL)(1.0 / rho);
    const REAL c0 = (REAL)(2.0 / (1.0 + a));
    F(hso_spmv)(n, rp, ci, v, x, tmp);                               /* :287 */
    for (int32_t i = 0; i < n; ++i) {                               /* :237-244 */
        REAL ri = (l1inv[i] * (b[i] - tmp[i])) * inv_rho;
        r[i] = ri;
        z[i] = c0 * ri;
    }
    double rho_s = (1.0 - a) / (1.0 + a);                            /* :296 */
    for (int32_t k = 1; k <= degree; ++k) {
        for (int32_t i = 0; i < n; ++i) x[i] += z[i];               /* :300, :67-70 */
        if (k < degree) {
            F(hso_spmv)(n, rp, ci, v, z, tmp);                       /* :305 */
            for (int32_t i = 0; i < n; ++i)                          /* :247-250 */
                r[i] = r[i] - (l1inv[i] * tmp[i]) * inv_rho;
            double rho_new = 1.0 / (2.0 * (1.0 + a) / (1.0 - a) - rho_s); /* :311 */
            const REAL c1 = (REAL)(rho_new * rho_s);
            const REAL c2 = (REAL)(4.0 * rho_new / (1.0 - a));
            for (int32_t i = 0; i < n; ++i) z[i] = c1 * z[i] + c2 * r[i]; /* :253-256 */
            rho_s = rho_new;
        }
    }
}

#undef F
#undef CAT2
#undef CAT2_
