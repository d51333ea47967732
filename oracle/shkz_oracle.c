/*
 * shkz_oracle.c -- CPU restatement of the reference MAC pressure projection.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA path: only
 * the test suite, the smoke check and the CPU-baseline leg of the benchmark
 * load it. The product library never links or calls it.
 *
 * It restates, in plain C with the same double-precision operation order:
 *   - face solid areas  macutility3::compute_area_fraction
 *                       (src/utility/macutility3.cpp:98-171) and
 *                       utility::get_area (include/shiokaze/utility/utility.h:191-226)
 *   - face liquid rhos  macutility3::compute_fluid_fraction (macutility3.cpp:172-200),
 *                       utility::fraction (utility.h:174-182)
 *   - unknown labelling mark_body (src/projection/macpressuresolver3.cpp:130-167),
 *                       numbered tile-major then x-fastest inside a tile
 *                       (src/array/tiledarray3.cpp:314-340, 806-825)
 *   - assembly          macpressuresolver3.cpp:179-216 into a row-sorted CSR
 *                       (RCMatrix::add_to_element keeps rows sorted,
 *                       src/math/RCMatrix.cpp:256-279)
 *   - PCG               PCGSolver::solve (local/include/pcgsolver/pcg_solver.h:246-295)
 *                       with either the identity (the preconditioner result is
 *                       discarded at pcg_solver.h:379-384) or the MIC(0)
 *                       factor and sweeps (pcg_solver.h:88-223) applied
 *   - velocity update   macpressuresolver3.cpp:262-284
 *   - FLIP splat        macnbflip3::splat over the pointgridhash3 edge hash
 *                       (src/flip/macnbflip3.cpp:103-148,
 *                       src/pointgridhash/pointgridhash3.cpp:90-100, 218-231)
 *                       and macflipliquid3's combined velocity
 *                       (src/liquid/macflipliquid3.cpp:135-151); see shkzo_splat
 *
 * Grids are dense, x fastest: cell (i,j,k) at i + nx*(j + ny*k); nodal grids
 * are (nx+1)*(ny+1)*(nz+1); face grid d has nx+(d==0), ny+(d==1), nz+(d==2).
 * Level-set inputs are the values the reference's array3::operator() returns
 * (stored value, fill value inside, background outside).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "shkz_oracle.h"

#define IDX(i, j, k, w, h) ((size_t)(i) + (size_t)(w) * ((size_t)(j) + (size_t)(h) * (size_t)(k)))

static inline int face_w(int nx, int d) { return nx + (d == 0); }
static inline int face_h(int ny, int d) { return ny + (d == 1); }
static inline int face_d(int nz, int d) { return nz + (d == 2); }
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* utility::get_area (utility.h:191-226): marching squares on the unit square
 * then the shoelace formula over the resulting point list. */
double shkzo_get_area(const double iso[2][2])
{
    static const int quads[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
    double v[4], p[8][2];
    int pnum = 0;
    for (int n = 0; n < 4; ++n) v[n] = iso[quads[n][0]][quads[n][1]];
    for (int n = 0; n < 4; ++n) {
        if (v[n] < 0.0) {
            p[pnum][0] = quads[n][0];
            p[pnum][1] = quads[n][1];
            pnum++;
        }
        if (v[n] * v[(n + 1) % 4] < 0) {
            double y0 = v[n], y1 = v[(n + 1) % 4];
            if (y0 - y1) {
                double a = y0 / (y0 - y1);
                const int *p0 = quads[n], *p1 = quads[(n + 1) % 4];
                p[pnum][0] = (1.0 - a) * p0[0] + a * p1[0];
                p[pnum][1] = (1.0 - a) * p0[1] + a * p1[1];
                pnum++;
            }
        }
    }
    double sum = 0.0;
    for (int m = 0; m < pnum; m++)
        sum += p[m][0] * p[(m + 1) % pnum][1] - p[m][1] * p[(m + 1) % pnum][0];
    return 0.5 * sum;
}

/* utility::fraction (utility.h:174-182) */
double shkzo_fraction(double phi0, double phi1)
{
    if (phi0 * phi1 >= 0.0) {
        if (phi0 < 0.0 || phi1 < 0.0) return 1.0;
        return 0.0;
    }
    double d = fabs(phi1 - phi0);
    if (d < DBL_MIN) d = DBL_MIN;
    return -(phi0 < phi1 ? phi0 : phi1) / d;
}

/* levelset_exist (include/shiokaze/array/array_utility3.h:112-122): some
 * active value is negative. */
static int levelset_exist(const float *v, const unsigned char *active, size_t n)
{
    if (!active) return 0;
    for (size_t i = 0; i < n; ++i)
        if (active[i] && v[i] < 0.0f) return 1;
    return 0;
}

/* one of the four nodes of face (d; i,j,k) is active in the solid grid */
static int act_face(const unsigned char *solid_active, int nx, int ny, int d, int i, int j, int k)
{
    const int NX = nx + 1, NY = ny + 1;
    /* the face spans the two axes other than d */
    const int ax = d == 0 ? 1 : 0, ay = d == 2 ? 1 : 2;
    int act = 0;
    for (int b = 0; b < 2; ++b)
        for (int a = 0; a < 2; ++a) {
            int n[3] = {i, j, k};
            n[ax] += a;
            n[ay] += b;
            act |= solid_active[IDX(n[0], n[1], n[2], NX, NY)];
        }
    return act;
}

void shkzo_fractions(int nx, int ny, int nz,
                     const float *solid, const unsigned char *solid_active,
                     const float *fluid, const unsigned char *fluid_active,
                     double eps_solid, double eps_fluid,
                     int second_order_fluid, int second_order_solid,
                     float *area[3], float *rho[3], float *const density[3])
{
    const int NX = nx + 1, NY = ny + 1;
    const size_t nn = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    const int solid_exists = levelset_exist(solid, solid_active, nn);
    const int fluid_exists = levelset_exist(fluid, fluid_active, (size_t)nx * ny * nz);
    for (int d = 0; d < 3; ++d) {
        const int fw = face_w(nx, d), fh = face_h(ny, d), fd = face_d(nz, d);
        const int nd = d == 0 ? nx : (d == 1 ? ny : nz);
        for (int k = 0; k < fd; ++k)
            for (int j = 0; j < fh; ++j)
                for (int i = 0; i < fw; ++i) {
                    const size_t f = IDX(i, j, k, fw, fh);
                    const int pd = d == 0 ? i : (d == 1 ? j : k);
                    /* --- solid area (macutility3.cpp:98-171) --- */
                    double a;
                    if (!solid_exists) {
                        a = (pd == 0 || pd == nd) ? 0.0 : 1.0; /* clear(1.0) + closed walls :158-170 */
                    } else {
                        int ni[4][3];
                        /* quadsolid[0][0], [1][0], [1][1], [0][1] (:120-136) */
                        if (d == 0) {
                            int t[4][3] = {{i, j, k}, {i, j + 1, k}, {i, j + 1, k + 1}, {i, j, k + 1}};
                            memcpy(ni, t, sizeof t);
                        } else if (d == 1) {
                            int t[4][3] = {{i, j, k}, {i + 1, j, k}, {i + 1, j, k + 1}, {i, j, k + 1}};
                            memcpy(ni, t, sizeof t);
                        } else {
                            int t[4][3] = {{i, j, k}, {i + 1, j, k}, {i + 1, j + 1, k}, {i, j + 1, k}};
                            memcpy(ni, t, sizeof t);
                        }
                        /* the face is active in the areas grid when one of its
                         * four nodes is active in the solid grid (:104-118) */
                        int act = 0;
                        double q[2][2];
                        for (int c = 0; c < 4; ++c) {
                            size_t nidx = IDX(ni[c][0], ni[c][1], ni[c][2], NX, NY);
                            act |= solid_active[nidx];
                        }
                        q[0][0] = solid[IDX(ni[0][0], ni[0][1], ni[0][2], NX, NY)];
                        q[1][0] = solid[IDX(ni[1][0], ni[1][1], ni[1][2], NX, NY)];
                        q[1][1] = solid[IDX(ni[2][0], ni[2][1], ni[2][2], NX, NY)];
                        q[0][1] = solid[IDX(ni[3][0], ni[3][1], ni[3][2], NX, NY)];
                        if (act) {
                            if (pd == 0 || pd == nd) a = 0.0;
                            else a = 1.0 - shkzo_get_area(q);
                            if (a && a < eps_solid) a = eps_solid;
                        } else {
                            /* inactive face: the flood-filled value (1 outside
                             * the solid, background 0 inside). With all four
                             * nodes on one side of a banded level set this is
                             * exactly 1 - get_area. */
                            a = 1.0 - shkzo_get_area(q);
                        }
                    }
                    float af = (float)a;
                    if (density && solid_exists && act_face(solid_active, nx, ny, d, i, j, k)) {
                        /* set_solid_density: active faces of the area grid become
                         * density*area + (1 - density) (macpressuresolver3.cpp:75-80) */
                        const float dens = density[d][f];
                        const float da = dens * af;
                        af = (float)((double)da + (1.0 - (double)dens));
                    }
                    if (!second_order_solid && af) af = 1.0f; /* macpressuresolver3.cpp:89-93 */
                    area[d][f] = af;
                    /* --- liquid fraction (macutility3.cpp:172-200) --- */
                    double r;
                    if (!fluid_exists) {
                        r = 1.0;
                    } else {
                        int ci = clampi(i, 0, nx - 1), cj = clampi(j, 0, ny - 1), ck = clampi(k, 0, nz - 1);
                        int bi = clampi(i - (d == 0), 0, nx - 1), bj = clampi(j - (d == 1), 0, ny - 1),
                            bk = clampi(k - (d == 2), 0, nz - 1);
                        r = shkzo_fraction(fluid[IDX(ci, cj, ck, nx, ny)], fluid[IDX(bi, bj, bk, nx, ny)]);
                        if (r && r < eps_fluid) r = eps_fluid;
                    }
                    float rf = (float)r;
                    if (!second_order_fluid && rf) rf = 1.0f; /* macpressuresolver3.cpp:83-87 */
                    rho[d][f] = rf;
                }
    }
}

/* mark_body (macpressuresolver3.cpp:134-158) for one cell. */
static int is_unknown(int nx, int ny, int nz, const float *fluid, float *const area[3], float *const rho[3],
                      int i, int j, int k)
{
    if (!(fluid[IDX(i, j, k, nx, ny)] < 0.0f)) return 0;
    const int q[6][3] = {{i + 1, j, k}, {i - 1, j, k}, {i, j + 1, k}, {i, j - 1, k}, {i, j, k + 1}, {i, j, k - 1}};
    const int fc[6][3] = {{i + 1, j, k}, {i, j, k}, {i, j + 1, k}, {i, j, k}, {i, j, k + 1}, {i, j, k}};
    for (int nq = 0; nq < 6; ++nq) {
        if (q[nq][0] < 0 || q[nq][1] < 0 || q[nq][2] < 0 || q[nq][0] >= nx || q[nq][1] >= ny || q[nq][2] >= nz)
            continue;
        if (fluid[IDX(q[nq][0], q[nq][1], q[nq][2], nx, ny)] < 0.0f) {
            const int d = nq / 2;
            const size_t f = IDX(fc[nq][0], fc[nq][1], fc[nq][2], face_w(nx, d), face_h(ny, d));
            if (area[d][f] && rho[d][f]) return 1;
        }
    }
    return 0;
}

long long shkzo_label(int nx, int ny, int nz, int tile, const float *fluid,
                      float *const area[3], float *const rho[3], long long *index)
{
    const int bx = (nx + tile - 1) / tile, by = (ny + tile - 1) / tile, bz = (nz + tile - 1) / tile;
    long long count = 0;
    for (size_t c = 0; c < (size_t)nx * ny * nz; ++c) index[c] = -1;
    /* const_serial_inside/all visit tiles in bi + bx*(bj + by*bk) order and
     * cells x-fastest inside a tile (tiledarray3.cpp:314-340, 490-492) */
    for (int tk = 0; tk < bz; ++tk)
        for (int tj = 0; tj < by; ++tj)
            for (int ti = 0; ti < bx; ++ti) {
                const int oi = ti * tile, oj = tj * tile, ok = tk * tile;
                const int zx = nx - oi < tile ? nx - oi : tile;
                const int zy = ny - oj < tile ? ny - oj : tile;
                const int zz = nz - ok < tile ? nz - ok : tile;
                for (int kk = 0; kk < zz; ++kk)
                    for (int jj = 0; jj < zy; ++jj)
                        for (int ii = 0; ii < zx; ++ii) {
                            const int i = oi + ii, j = oj + jj, k = ok + kk;
                            if (is_unknown(nx, ny, nz, fluid, area, rho, i, j, k))
                                index[IDX(i, j, k, nx, ny)] = count++;
                        }
            }
    return count;
}

/* Row insertion keeping columns sorted; entries summing to zero are removed
 * (RCMatrix::add_to_element, src/math/RCMatrix.cpp:256-279). */
static void row_add(long long *cols, double *vals, int *len, long long col, double v)
{
    int n = *len, p = 0;
    while (p < n && cols[p] < col) ++p;
    if (p < n && cols[p] == col) {
        vals[p] += v;
        if (vals[p] == 0.0) {
            memmove(cols + p, cols + p + 1, sizeof(long long) * (n - p - 1));
            memmove(vals + p, vals + p + 1, sizeof(double) * (n - p - 1));
            *len = n - 1;
        }
        return;
    }
    memmove(cols + p + 1, cols + p, sizeof(long long) * (n - p));
    memmove(vals + p + 1, vals + p, sizeof(double) * (n - p));
    cols[p] = col;
    vals[p] = v;
    *len = n + 1;
}

long long shkzo_assemble(int nx, int ny, int nz, double dx, double dt, const float *fluid,
                         float *const area[3], float *const rho[3],
                         float *const velocity[3], float *const solid_velocity[3],
                         const long long *index, long long n_unknowns,
                         long long *indptr, long long *indices, double *data, double *rhs)
{
    /* assembly of one row (macpressuresolver3.cpp:179-216) */
    long long *rcols = (long long *)malloc(sizeof(long long) * 7 * (size_t)(n_unknowns > 0 ? n_unknowns : 1));
    double *rvals = (double *)malloc(sizeof(double) * 7 * (size_t)(n_unknowns > 0 ? n_unknowns : 1));
    int *rlen = (int *)calloc((size_t)(n_unknowns > 0 ? n_unknowns : 1), sizeof(int));
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const long long row = index[IDX(i, j, k, nx, ny)];
                if (row < 0) continue;
                long long *cols = rcols + 7 * row;
                double *vals = rvals + 7 * row;
                double b = 0.0;
                const int q[6][3] = {{i + 1, j, k}, {i - 1, j, k}, {i, j + 1, k}, {i, j - 1, k}, {i, j, k + 1}, {i, j, k - 1}};
                const int fc[6][3] = {{i + 1, j, k}, {i, j, k}, {i, j + 1, k}, {i, j, k}, {i, j, k + 1}, {i, j, k}};
                const int sgn[6] = {1, -1, 1, -1, 1, -1};
                double diagonal = 0.0;
                for (int nq = 0; nq < 6; ++nq) {
                    const int d = nq / 2;
                    const size_t f = IDX(fc[nq][0], fc[nq][1], fc[nq][2], face_w(nx, d), face_h(ny, d));
                    const double a = area[d][f];
                    const int oob = q[nq][0] < 0 || q[nq][1] < 0 || q[nq][2] < 0 ||
                                    q[nq][0] >= nx || q[nq][1] >= ny || q[nq][2] >= nz;
                    if (!oob && a) {
                        const double r = rho[d][f];
                        if (r) {
                            const double value = dt * a / (dx * dx * r);
                            const size_t qc = IDX(q[nq][0], q[nq][1], q[nq][2], nx, ny);
                            if (fluid[qc] < 0.0f) row_add(cols, vals, &rlen[row], index[qc], -value);
                            diagonal += value;
                        }
                    }
                    b += -sgn[nq] * a * velocity[d][f] / dx;
                    if (a < 1.0) {
                        const double u = solid_velocity ? solid_velocity[d][f] : 0.0f;
                        b += -sgn[nq] * (1.0 - a) * u / dx;
                    }
                }
                row_add(cols, vals, &rlen[row], row, diagonal);
                rhs[row] = b;
            }
    long long nnz = 0;
    for (long long r = 0; r < n_unknowns; ++r) {
        indptr[r] = nnz;
        for (int e = 0; e < rlen[r]; ++e) {
            indices[nnz] = rcols[7 * r + e];
            data[nnz] = rvals[7 * r + e];
            ++nnz;
        }
    }
    indptr[n_unknowns] = nnz;
    free(rcols);
    free(rvals);
    free(rlen);
    return nnz;
}

/* ---------------------------------------------------------------------- */
/* MIC(0) in CSC lower form (factor_modified_incomplete_cholesky0,
 * pcg_solver.h:88-189). The matrix is symmetric, so column k of the lower
 * triangle is the upper part of CSR row k. */
typedef struct {
    long long n;
    long long *colstart, *rowindex;
    double *value, *invdiag, *adiag;
} mic0_factor;

static void mic0_build(long long n, const long long *indptr, const long long *indices, const double *data,
                       mic0_factor *F, double omega, double min_ratio)
{
    F->n = n;
    F->colstart = (long long *)malloc(sizeof(long long) * (n + 1));
    F->invdiag = (double *)calloc((size_t)n, sizeof(double));
    F->adiag = (double *)calloc((size_t)n, sizeof(double));
    long long cnt = 0;
    for (long long i = 0; i < n; ++i)
        for (long long p = indptr[i]; p < indptr[i + 1]; ++p)
            if (indices[p] > i) ++cnt;
    F->rowindex = (long long *)malloc(sizeof(long long) * (cnt > 0 ? cnt : 1));
    F->value = (double *)malloc(sizeof(double) * (cnt > 0 ? cnt : 1));
    cnt = 0;
    for (long long i = 0; i < n; ++i) {
        F->colstart[i] = cnt;
        for (long long p = indptr[i]; p < indptr[i + 1]; ++p) {
            if (indices[p] > i) {
                F->rowindex[cnt] = indices[p];
                F->value[cnt] = data[p];
                ++cnt;
            } else if (indices[p] == i) {
                F->invdiag[i] = F->adiag[i] = data[p];
            }
        }
    }
    F->colstart[n] = cnt;
    for (long long k = 0; k < n; ++k) {
        if (F->adiag[k] == 0) continue;
        if (F->invdiag[k] < min_ratio * F->adiag[k]) F->invdiag[k] = 1 / sqrt(F->adiag[k]);
        else F->invdiag[k] = 1 / sqrt(F->invdiag[k]);
        for (long long p = F->colstart[k]; p < F->colstart[k + 1]; ++p) F->value[p] *= F->invdiag[k];
        for (long long p = F->colstart[k]; p < F->colstart[k + 1]; ++p) {
            const long long j = F->rowindex[p];
            const double multiplier = F->value[p];
            double missing = 0;
            long long a = F->colstart[k];
            long long b = 0;
            const long long rj0 = indptr[j], rjn = indptr[j + 1] - indptr[j];
            while (a < F->colstart[k + 1] && F->rowindex[a] < j) {
                while (b < rjn) {
                    if (indices[rj0 + b] < F->rowindex[a]) ++b;
                    else if (indices[rj0 + b] == F->rowindex[a]) break;
                    else { missing += F->value[a]; break; }
                }
                ++a;
            }
            if (a < F->colstart[k + 1] && F->rowindex[a] == j) F->invdiag[j] -= multiplier * F->value[a];
            ++a;
            b = F->colstart[j];
            while (a < F->colstart[k + 1] && b < F->colstart[j + 1]) {
                if (F->rowindex[b] < F->rowindex[a]) ++b;
                else if (F->rowindex[b] == F->rowindex[a]) {
                    F->value[b] -= multiplier * F->value[a];
                    ++a;
                    ++b;
                } else {
                    missing += F->value[a];
                    ++a;
                }
            }
            while (a < F->colstart[k + 1]) {
                missing += F->value[a];
                ++a;
            }
            F->invdiag[j] -= omega * multiplier * missing;
        }
    }
}

static void mic0_free(mic0_factor *F)
{
    free(F->colstart); free(F->rowindex); free(F->value); free(F->invdiag); free(F->adiag);
}

/* solve_lower then solve_lower_transpose_in_place (pcg_solver.h:195-223) */
static void mic0_apply(const mic0_factor *F, const double *rhs, double *out)
{
    const long long n = F->n;
    memcpy(out, rhs, sizeof(double) * n);
    for (long long i = 0; i < n; ++i) {
        out[i] *= F->invdiag[i];
        for (long long j = F->colstart[i]; j < F->colstart[i + 1]; ++j) out[F->rowindex[j]] -= F->value[j] * out[i];
    }
    long long i = n;
    if (n == 0) return;
    do {
        --i;
        for (long long j = F->colstart[i]; j < F->colstart[i + 1]; ++j) out[i] -= F->value[j] * out[F->rowindex[j]];
        out[i] *= F->invdiag[i];
    } while (i != 0);
}

void shkzo_mic0_apply(long long n, const long long *indptr, const long long *indices, const double *data,
                      double omega, double min_ratio, const double *r, double *z, double *invdiag_out)
{
    mic0_factor F;
    mic0_build(n, indptr, indices, data, &F, omega, min_ratio);
    mic0_apply(&F, r, z);
    if (invdiag_out) memcpy(invdiag_out, F.invdiag, sizeof(double) * n);
    mic0_free(&F);
}

void shkzo_spmv(long long n, const long long *indptr, const long long *indices, const double *data,
                const double *x, double *y)
{
    /* FixedSparseMatrix multiply (local/include/pcgsolver/sparse_matrix.h:265-275) */
    for (long long i = 0; i < n; ++i) {
        double s = 0;
        for (long long p = indptr[i]; p < indptr[i + 1]; ++p) s += data[p] * x[indices[p]];
        y[i] = s;
    }
}

static double dot(long long n, const double *a, const double *b)
{ double s = 0.0; for (long long i = 0; i < n; ++i) s += a[i] * b[i]; return s; }
static void axpy(long long n, double a, const double *x, double *y)
{ for (long long i = 0; i < n; ++i) y[i] += a * x[i]; }
static double abs_max(long long n, const double *x)
{
    /* fabs(x[idamax]) with the first maximal index (blas_wrapper.h:77-96) */
    long long k = 0; double m = -1.0;
    for (long long i = 0; i < n; ++i) { double a = fabs(x[i]); if (a > m) { m = a; k = i; } }
    return n ? fabs(x[k]) : 0.0;
}

int shkzo_pcg(long long n, const long long *indptr, const long long *indices, const double *data,
              const double *rhs, double *x, double tol, int max_iterations, int use_mic0,
              double omega, double min_ratio, double *reresid_out)
{
    /* PCGSolver::solve (pcg_solver.h:246-295) */
    double *z = (double *)malloc(sizeof(double) * (n ? n : 1));
    double *s = (double *)malloc(sizeof(double) * (n ? n : 1));
    double *r = (double *)malloc(sizeof(double) * (n ? n : 1));
    mic0_factor F;
    int built = 0, iterations = 0;
    memset(x, 0, sizeof(double) * n);
    memcpy(r, rhs, sizeof(double) * n);
    double residual = abs_max(n, r);
    const double residual0 = residual;
    if (residual == 0) { *reresid_out = 0; iterations = 0; goto done; }
    {
        const double abs_tol = tol * residual;
        if (use_mic0) { mic0_build(n, indptr, indices, data, &F, omega, min_ratio); built = 1; mic0_apply(&F, r, z); }
        else memcpy(z, r, sizeof(double) * n);
        double rho = dot(n, z, r);
        if (rho == 0 || rho != rho) { *reresid_out = residual; iterations = 0; goto done; }
        memcpy(s, z, sizeof(double) * n);
        int it;
        for (it = 0; it < max_iterations; ++it) {
            shkzo_spmv(n, indptr, indices, data, s, z);
            const double alpha = rho / dot(n, s, z);
            axpy(n, alpha, s, x);
            axpy(n, -alpha, z, r);
            residual = abs_max(n, r);
            if (residual <= abs_tol) {
                iterations = it + 1;
                *reresid_out = residual / residual0;
                goto done;
            }
            if (use_mic0) mic0_apply(&F, r, z);
            else memcpy(z, r, sizeof(double) * n);
            const double rho_new = dot(n, z, r);
            const double beta = rho_new / rho;
            for (long long i = 0; i < n; ++i) z[i] += beta * s[i];
            { double *t = s; s = z; z = t; }
            rho = rho_new;
        }
        iterations = it;
        *reresid_out = residual / residual0;
    }
done:
    if (built) mic0_free(&F);
    free(z); free(s); free(r);
    return iterations;
}

void shkzo_update_velocity(int nx, int ny, int nz, double dx, double dt, const float *pressure,
                           float *const area[3], float *const rho[3], float *const solid_velocity[3],
                           float *velocity[3], unsigned char *velocity_active[3], float *const density[3])
{
    /* macpressuresolver3.cpp:269-284; pressure is the float grid m_pressure
     * (0 = background where no unknown was written). */
    for (int d = 0; d < 3; ++d) {
        const int fw = face_w(nx, d), fh = face_h(ny, d), fd = face_d(nz, d);
        const int nd = d == 0 ? nx : (d == 1 ? ny : nz);
        for (int k = 0; k < fd; ++k)
            for (int j = 0; j < fh; ++j)
                for (int i = 0; i < fw; ++i) {
                    const size_t f = IDX(i, j, k, fw, fh);
                    if (!velocity_active[d][f]) continue;
                    const double r = rho[d][f];
                    const int pd = d == 0 ? i : (d == 1 ? j : k);
                    const double solid_u = solid_velocity ? solid_velocity[d][f] : 0.0f;
                    if (area[d][f] && r) {
                        if (pd == 0 || pd == nd) velocity[d][f] = (float)solid_u;
                        else {
                            const float p1 = pressure[IDX(i, j, k, nx, ny)];
                            const float p0 = pressure[IDX(i - (d == 0), j - (d == 1), k - (d == 2), nx, ny)];
                            const float diff = +p1 - p0;
                            const float value = (float)(dt * diff / (r * dx));
                            velocity[d][f] = velocity[d][f] - value;
                        }
                        if (density) {
                            /* macpressuresolver3.cpp:286-293 */
                            const float scale = (float)(1.0 - (1.0 - (double)area[d][f]) * (double)density[d][f]);
                            velocity[d][f] = scale * velocity[d][f];
                        }
                    } else {
                        velocity[d][f] = 0.0f; /* set_off: inactive, reads background 0 */
                        velocity_active[d][f] = 0;
                    }
                }
    }
}

/* ------------------------------------------------------------------------
 * FLIP splat before the projection.
 *
 * Particles are records of `stride` bytes in the reference's layout
 * (macnbflip3::Particle, src/flip/macnbflip3.h:128-139): float p[3] at
 * off_p, float velocity[3] at off_v, float mass at off_m, float c[3][3] at
 * off_c (off_c < 0: APIC off), char bullet at off_bullet (< 0: none).
 *
 * Restates, with the reference's operation order and types:
 *   - the edge hash  pointgridhash3::sort_points, EDGE_MODE
 *                    (src/pointgridhash/pointgridhash3.cpp:90-100): every
 *                    particle goes, in index order, into the bucket
 *                    shape3::find_edge(p/dx, dim) (include/shiokaze/math/
 *                    shape.h:748-750: (p/dx) rounded to float, + 0.5 off the
 *                    edge axis rounded to float, truncated, clamped)
 *   - macnbflip3::splat (src/flip/macnbflip3.cpp:103-148): faces touched by
 *                    a splatting particle (8 per dim, clamped to the CELL
 *                    shape) are activated; each then sums over
 *                    get_face_neighbors(face, dim) (pointgridhash3.cpp:
 *                    218-231), whose loops run ri, rj, rk over {0,1} for all
 *                    three axes, so along the face's own axis each bucket is
 *                    visited twice and every particle is counted twice
 *   - the combined grid velocity (src/liquid/macflipliquid3.cpp:135-151).
 * Outputs: mass/momentum/splat_active per face (the splat grid; faces with
 * zero mass are switched off), velocity/velocity_active updated in place. */
static inline float rd_f(const unsigned char *rec, int off, int k)
{
    float v;
    memcpy(&v, rec + off + 4 * k, 4);
    return v;
}

static inline int edge_axis(float pc, double dx, int half, int extent)
{
    const float q = (float)((double)pc / dx);
    const float t = (float)((double)q + (half ? 0.5 : 0.0));
    return clampi((int)t, 0, extent - 1);
}

static inline double tent(double r, double dx)
{
    const double x = fabs(r) / dx;
    const double v = 1.0 - x;
    return 0.0 < v ? v : 0.0;
}

int shkzo_splat(int nx, int ny, int nz, double dx, long long count, const void *particles, int stride,
                int off_p, int off_v, int off_m, int off_c, int off_bullet, int splat_bullet,
                float *velocity[3], unsigned char *velocity_active[3],
                float *mass[3], float *momentum[3], unsigned char *splat_active[3])
{
    const unsigned char *base = (const unsigned char *)particles;
    const int n3[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d) {
        const int fw = face_w(nx, d), fh = face_h(ny, d), fd = face_d(nz, d);
        const size_t nf = (size_t)fw * fh * fd;
        int E[3];
        for (int c = 0; c < 3; ++c) E[c] = n3[c] + (c != d);
        const size_t ne = (size_t)E[0] * E[1] * E[2];
        /* edge buckets as a counting sort that keeps index order */
        long long *start = (long long *)calloc(ne + 1, sizeof(long long));
        long long *key = (long long *)malloc(sizeof(long long) * (count ? count : 1));
        long long *list = (long long *)malloc(sizeof(long long) * (count ? count : 1));
        if (!start || !key || !list) { free(start); free(key); free(list); return -1; }
        for (long long n = 0; n < count; ++n) {
            const unsigned char *rec = base + (size_t)n * stride;
            int e[3];
            for (int c = 0; c < 3; ++c) e[c] = edge_axis(rd_f(rec, off_p, c), dx, c != d, E[c]);
            key[n] = (long long)IDX(e[0], e[1], e[2], E[0], E[1]);
            start[key[n] + 1]++;
        }
        for (size_t b = 0; b < ne; ++b) start[b + 1] += start[b];
        {
            long long *fill = (long long *)malloc(sizeof(long long) * (ne ? ne : 1));
            if (!fill) { free(start); free(key); free(list); return -1; }
            memcpy(fill, start, sizeof(long long) * ne);
            for (long long n = 0; n < count; ++n) list[fill[key[n]]++] = n;
            free(fill);
        }
        /* activation (macnbflip3.cpp:109-120) */
        memset(splat_active[d], 0, nf);
        for (long long n = 0; n < count; ++n) {
            const unsigned char *rec = base + (size_t)n * stride;
            if (!splat_bullet && off_bullet >= 0 && rec[off_bullet]) continue;
            int pi[3];
            for (int c = 0; c < 3; ++c) pi[c] = (int)((double)rd_f(rec, off_p, c) / dx - 0.5 * (d != c));
            for (int ii = 0; ii <= 1; ++ii)
                for (int jj = 0; jj <= 1; ++jj)
                    for (int kk = 0; kk <= 1; ++kk) {
                        const int i = clampi(pi[0] + ii, 0, nx - 1);
                        const int j = clampi(pi[1] + jj, 0, ny - 1);
                        const int k = clampi(pi[2] + kk, 0, nz - 1);
                        splat_active[d][IDX(i, j, k, fw, fh)] = 1;
                    }
        }
        /* gather (macnbflip3.cpp:121-143) */
        for (int k = 0; k < fd; ++k)
            for (int j = 0; j < fh; ++j)
                for (int i = 0; i < fw; ++i) {
                    const size_t f = IDX(i, j, k, fw, fh);
                    mass[d][f] = 0.0f;
                    momentum[d][f] = 0.0f;
                    if (!splat_active[d][f]) continue;
                    const int fi[3] = {i, j, k};
                    double pos[3];
                    for (int c = 0; c < 3; ++c) pos[c] = ((double)fi[c] + 0.5 * (d != c)) * dx;
                    float mom = 0.0f, m = 0.0f;
                    for (int dir = -1; dir <= 0; ++dir)
                        for (int ri = 0; ri <= 1; ++ri)
                            for (int rj = 0; rj <= 1; ++rj)
                                for (int rk = 0; rk <= 1; ++rk) {
                                    const int r3[3] = {ri, rj, rk};
                                    int q[3];
                                    int out = 0;
                                    for (int c = 0; c < 3; ++c) {
                                        q[c] = fi[c] + (c != d) * r3[c] + (c == d) * dir;
                                        out |= q[c] < 0 || q[c] >= E[c];
                                    }
                                    if (out) continue;
                                    const size_t b = IDX(q[0], q[1], q[2], E[0], E[1]);
                                    for (long long s = start[b]; s < start[b + 1]; ++s) {
                                        const unsigned char *rec = base + (size_t)list[s] * stride;
                                        if (!splat_bullet && off_bullet >= 0 && rec[off_bullet]) continue;
                                        float r[3];
                                        for (int c = 0; c < 3; ++c) r[c] = (float)((double)rd_f(rec, off_p, c) - pos[c]);
                                        const double w = tent(r[0], dx) * tent(r[1], dx) * tent(r[2], dx);
                                        if (w != 0.0) {
                                            const double pm = (double)rd_f(rec, off_m, 0);
                                            mom = (float)((double)mom + w * pm * (double)rd_f(rec, off_v, d));
                                            m = (float)((double)m + w * pm);
                                            if (off_c >= 0) {
                                                double dot = 0.0;
                                                for (int c = 0; c < 3; ++c)
                                                    dot += (double)rd_f(rec, off_c, 3 * d + c) *
                                                           (pos[c] - (double)rd_f(rec, off_p, c));
                                                mom = (float)((double)mom + w * pm * dot);
                                            }
                                        }
                                    }
                                }
                    if (m != 0.0f) {
                        mass[d][f] = m;
                        momentum[d][f] = mom;
                    } else {
                        splat_active[d][f] = 0;
                    }
                }
        free(start); free(key); free(list);
        /* combined grid velocity (macflipliquid3.cpp:141-150) */
        for (size_t f = 0; f < nf; ++f) {
            if (!splat_active[d][f]) continue;
            const double gm64 = 1.0 - (double)mass[d][f];
            const float gm = velocity_active[d][f] ? (float)(0.0 < gm64 ? gm64 : 0.0) : 0.0f;
            const float num = gm * velocity[d][f] + momentum[d][f];
            const float den = gm + mass[d][f];
            velocity[d][f] = num / den;
            velocity_active[d][f] = 1;
        }
    }
    return 0;
}
