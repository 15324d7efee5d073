/*
 * pd_oracle.c -- CPU FP64 restatement of PeriDyn's per-step force path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; never part of the product).
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 *
 * Each function cites the reference file:line it restates (paths are
 * relative to the PeriDyn source tree, src/).  Index arithmetic is 1-based
 * in the data (family entries, neighbour lists) exactly as in Julia; the C
 * loops themselves are 0-based.
 *
 * Parity unpinned by the reference itself: the reference is Julia (not
 * available here) and ships no tests or golden vectors, so this
 * restatement is pinned by analytical known answers instead (homogeneous
 * stretch, lattice neighbour counts, momentum and energy conservation of
 * the bond, state-based and contact terms).
 */
#include "pd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define COL(a, ld, r, c) ((a)[(size_t)(c) * (size_t)(ld) + (size_t)(r)])

/* ------------------------------------------------------------------ */
/* Julia scalar helpers                                                 */
/* ------------------------------------------------------------------ */

/* Julia Base.mod(x::Float64, y::Float64). */
static double jl_mod(double x, double y) {
    if (isinf(y) && isfinite(x)) return x;
    double r = fmod(x, y); /* Julia rem(x, y) for IEEE floats is exact fmod */
    if (r == 0.0) return copysign(r, y);
    if ((r > 0) != (y > 0)) return r + y;
    return r;
}

/* Julia fld(x, y) = div(x, y, RoundDown) = round((x - mod(x, y)) / y). */
double or_fld(double x, double y) {
    double r = jl_mod(x, y);
    return nearbyint((x - r) / y); /* round-half-even, default FP env */
}

/* Julia base/math.jl pow_body(x::Float64, n::Integer): compensated
 * repeated squaring.  muladd is fused on FMA hardware. */
static double jl_pow_body(double x, int64_t n) {
    double y = 1.0, xnlo = 0.0, ynlo = 0.0;
    if (n == 3) return x * x * x;
    if (n < 0) {
        double rx = 1.0 / x;
        if (n == -2) return rx * rx;
        if (isfinite(x)) xnlo = -fma(x, rx, -1.0) * rx;
        x = rx;
        n = -n;
    }
    while (n > 1) {
        if (n & 1) {
            double err = fma(y, xnlo, x * ynlo);
            double p = x * y;
            ynlo = fma(x, y, -p);
            y = p;
            ynlo += err;
        }
        double err = x * 2 * xnlo;
        double p = x * x;
        xnlo = fma(x, x, -p);
        x = p;
        xnlo += err;
        n >>= 1;
    }
    double err = fma(y, xnlo, x * ynlo);
    return (isfinite(x) && isfinite(err)) ? fma(x, y, err) : x * y;
}

/* Julia ^(x::Float64, y::Float64) for the cases used here. */
double or_pow(double x, double y) {
    if (x == 1.0) return 1.0;
    if (isnan(y)) return y;
    if (fabs(y) < 0x1.8p62) {
        int64_t yi = (int64_t)y;
        if ((double)yi == y) {
            if (yi == 0) return 1.0;
            return jl_pow_body(x, yi);
        }
    }
    return pow(x, y); /* non-integral exponent: libm (may differ by 1 ulp) */
}

/* const_macros.jl:113-134 get_magnitude (3-D): sqrt(a1*a1 + a2*a2 + a3*a3) */
static inline double mag3(double a1, double a2, double a3) {
    return sqrt(a1 * a1 + a2 * a2 + a3 * a3);
}

/* ------------------------------------------------------------------ */
/* Cell lists: peri.jl:459-520                                          */
/* ------------------------------------------------------------------ */

typedef struct {
    int64_t N[3];
    int64_t ncells;
    int64_t *start; /* ncells+1 CSR offsets into idx */
    int64_t *idx;   /* particle indices (0-based), ascending within a cell */
} cells_t;

/* peri.jl:484-486 cell_number (1-based in, 1-based out) */
static inline int64_t cell_number(int64_t i, int64_t j, int64_t k, const int64_t *N) {
    return i + (j - 1) * N[0] + (k - 1) * N[0] * N[1];
}

/* peri.jl:500-520 get_cells(x, horizon; max_part).  The cell a particle is
 * pushed into is clamp(fld(x - min, h), 1, max_part) per dimension. */
static void get_cells(int64_t n, const double *x, double h, int64_t max_part,
                      cells_t *c, int64_t *cell_of) {
    double mn[3], mx[3];
    for (int d = 0; d < 3; ++d) {
        mn[d] = INFINITY;
        mx[d] = -INFINITY;
    }
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            double v = x[3 * i + d];
            if (v < mn[d]) mn[d] = v;
            if (v > mx[d]) mx[d] = v;
        }
    for (int d = 0; d < 3; ++d) {
        double q = or_fld(mx[d] - mn[d], h);
        double v = fmax(1.0, fmin((double)max_part, q));
        c->N[d] = (int64_t)v;
    }
    c->ncells = c->N[0] * c->N[1] * c->N[2];
    int64_t *cnt = (int64_t *)calloc((size_t)c->ncells + 1, sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) {
        int64_t ijk[3];
        for (int d = 0; d < 3; ++d) {
            double q = or_fld(x[3 * i + d] - mn[d], h);
            ijk[d] = (int64_t)fmax(1.0, fmin((double)max_part, q));
        }
        int64_t cn = cell_number(ijk[0], ijk[1], ijk[2], c->N) - 1;
        cell_of[i] = cn;
        cnt[cn + 1]++;
    }
    for (int64_t k = 0; k < c->ncells; ++k) cnt[k + 1] += cnt[k];
    c->start = cnt;
    c->idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t *fill = (int64_t *)calloc((size_t)c->ncells, sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) { /* push! in ascending i order */
        int64_t cn = cell_of[i];
        c->idx[c->start[cn] + fill[cn]++] = i;
    }
    free(fill);
}

static void free_cells(cells_t *c) {
    free(c->start);
    free(c->idx);
}

/* peri.jl:459-471 neigh_cells: the in-range cells of the 3x3x3 block, in
 * kk, jj, ii nesting order.  Returns count; out holds 0-based cell ids. */
static int neigh_cells(int64_t cn0, const int64_t *N, int64_t *out) {
    int64_t i = cn0 % N[0] + 1;
    int64_t j = (cn0 / N[0]) % N[1] + 1;
    int64_t k = cn0 / (N[0] * N[1]) + 1;
    int cnt = 0;
    for (int64_t kk = k - 1; kk <= k + 1; ++kk)
        for (int64_t jj = j - 1; jj <= j + 1; ++jj)
            for (int64_t ii = i - 1; ii <= i + 1; ++ii)
                if ((0 < ii * jj * kk) && (ii <= N[0]) && (jj <= N[1]) && (kk <= N[2]))
                    out[cnt++] = cell_number(ii, jj, kk, N) - 1;
    return cnt;
}

static int cmp_i64(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* ------------------------------------------------------------------ */
/* Family: peri.jl:533-576 and general_material.jl:85-90                */
/* ------------------------------------------------------------------ */
int or_cal_family(int64_t n, const double *x, double horizon, int64_t max_neigh,
                  int64_t *family_out, int64_t *rows_out) {
    /* cal_family: max_neigh = min(max_neigh, size(x, 2)) */
    int64_t Mn = max_neigh < n ? max_neigh : n;
    int64_t *fam = (int64_t *)calloc((size_t)(Mn > 0 ? Mn : 1) * (size_t)(n > 0 ? n : 1), sizeof(int64_t));
    int64_t *cell_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    cells_t c;
    get_cells(n, x, horizon, 30, &c, cell_of);
    int overflow = 0;
    int64_t nb[27];
    for (int64_t cell_i = 0; cell_i < c.ncells; ++cell_i) {
        int nn = neigh_cells(cell_i, c.N, nb);
        for (int64_t a = c.start[cell_i]; a < c.start[cell_i + 1]; ++a) {
            int64_t ca = c.idx[a];
            int64_t ind = 1;
            double a1 = x[3 * ca], b1 = x[3 * ca + 1], c1 = x[3 * ca + 2];
            for (int q = 0; q < nn; ++q) {
                int64_t cell = nb[q];
                for (int64_t b = c.start[cell]; b < c.start[cell + 1]; ++b) {
                    int64_t fa = c.idx[b];
                    double a2 = x[3 * fa], b2 = x[3 * fa + 1], c2 = x[3 * fa + 2];
                    if ((ca != fa) &&
                        (((a1 - a2) * (a1 - a2) + (b1 - b2) * (b1 - b2) + (c1 - c2) * (c1 - c2)) <
                         horizon * horizon)) {
                        if (ind > Mn) { /* family[ind, ca] out of bounds */
                            overflow = 1;
                        } else {
                            COL(fam, Mn, ind - 1, ca) = fa + 1;
                        }
                        ind += 1;
                    }
                }
            }
        }
    }
    free_cells(&c);
    free(cell_of);
    if (overflow) {
        free(fam);
        return 3;
    }
    /* sort each column ascending (zeros first) */
    int64_t maxcount = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t *col = fam + (size_t)i * (size_t)Mn;
        qsort(col, (size_t)Mn, sizeof(int64_t), cmp_i64);
        int64_t cnt = 0;
        for (int64_t r = 0; r < Mn; ++r) cnt += col[r] > 0;
        if (cnt > maxcount) maxcount = cnt;
    }
    /* general_material.jl:88-90: k = M - max(sum(intact)); family[end:-1:k, :] */
    int64_t k = Mn - maxcount;
    if (k < 1) {
        free(fam);
        return 3;
    }
    int64_t rows = Mn - k + 1;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t r = 0; r < rows; ++r)
            COL(family_out, rows, r, i) = COL(fam, Mn, Mn - 1 - r, i);
    *rows_out = rows;
    free(fam);
    return 0;
}

/* peri.jl:342-354 weighted_volume: m_i = sum w|X|^2 * 1 * V_j, w = 1/|X| */
void or_weighted_volume(int64_t n, const double *x, const double *vol,
                        int64_t M, const int64_t *family, double *m) {
    for (int64_t i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int64_t k = 0; k < M; ++k) {
            int64_t j = COL(family, M, k, i);
            if ((j > 0) & (i + 1 != j)) {
                int64_t jj = j - 1;
                double d1 = x[3 * jj] - x[3 * i], d2 = x[3 * jj + 1] - x[3 * i + 1],
                       d3 = x[3 * jj + 2] - x[3 * i + 2];
                double mg = mag3(d1, d2, d3);
                double w = 1 / mg;                       /* peri.jl:102-104 */
                acc = acc + w * (mg * mg) * 1.0 * vol[jj]; /* horizon_correction == 1 */
            }
        }
        m[i] = acc;
    }
}

/* peri.jl:155-172 dilatation! (CPU) */
void or_dilatation(int64_t n, const double *y, const double *x,
                   const uint8_t *intact, const int64_t *family, int64_t M,
                   const double *vol, const double *m, double *theta,
                   int nthreads) {
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1) if (nthreads > 1)
    for (int64_t i = 0; i < n; ++i) {
        double th = 0.0;
        double c_i = 3 / m[i];
        for (int64_t k = 0; k < M; ++k) {
            if (COL(intact, M, k, i) == 1) {
                int64_t j = COL(family, M, k, i) - 1;
                double X1 = x[3 * j] - x[3 * i], X2 = x[3 * j + 1] - x[3 * i + 1],
                       X3 = x[3 * j + 2] - x[3 * i + 2];
                double Y1 = y[3 * j] - y[3 * i], Y2 = y[3 * j + 1] - y[3 * i + 1],
                       Y3 = y[3 * j + 2] - y[3 * i + 2];
                double xij = mag3(X1, X2, X3);
                double yij = mag3(Y1, Y2, Y3);
                double extension = yij - xij;
                double w = 1 / mag3(X1, X2, X3);
                th = th + c_i * w * xij * extension * vol[j] * 1.0;
            }
        }
        theta[i] = th;
    }
}

/* general_material.jl:296-369 force_density_T! (CPU). */
void or_force_density_T(int kind, int64_t n, int64_t M, double *f,
                        const double *y, const double *x,
                        const int64_t *family, uint8_t *intact,
                        const int64_t *type_rel, int64_t ntypes,
                        const double *cs, const double *density,
                        const double *vol, const double *c,
                        const double *m, const double *theta,
                        const double *K, const double *G, int nthreads) {
    /* bond_based.jl:179-181,229: items = bond_stiffness; items[1] is its
     * first (linear index 1) element, used for every type pair. */
    const double c11 = (kind == 0) ? c[0] : 0.0;
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1) if (nthreads > 1)
    for (int64_t i = 0; i < n; ++i) {
        int64_t ti = type_rel[i];
        double _den_i = density[ti - 1];
        for (int64_t k = 0; k < M; ++k) {
            if (!COL(intact, M, k, i)) continue;
            int64_t j = COL(family, M, k, i) - 1;
            int64_t tj = type_rel[j];
            double _den_j = density[tj - 1];
            double X1 = x[3 * j] - x[3 * i], X2 = x[3 * j + 1] - x[3 * i + 1],
                   X3 = x[3 * j + 2] - x[3 * i + 2];
            double Y1 = y[3 * j] - y[3 * i], Y2 = y[3 * j + 1] - y[3 * i + 1],
                   Y3 = y[3 * j + 2] - y[3 * i + 2];
            double yij = mag3(Y1, Y2, Y3);
            double xij = mag3(X1, X2, X3);
            double extension = yij - xij;
            double s = extension / xij;
            size_t tp = (size_t)(ti - 1) + (size_t)(tj - 1) * (size_t)ntypes;
            if (s < cs[tp]) {
                double tij;
                if (kind == 0) {
                    tij = s * c11; /* bond_based.jl:195-197 */
                } else {
                    /* ordinary_state_based.jl:176-187 */
                    double wij = 1 / mag3(X1, X2, X3);
                    double wji = 1 / mag3(-X1, -X2, -X3);
                    double Kij = K[tp], Gij = G[tp];
                    double a = wij / m[i], b = wji / m[j];
                    tij = (3 * Kij - 5 * Gij) * (theta[i] * xij * a + theta[j] * xij * b) +
                          15 * Gij * extension * (a + b);
                }
                double xx = 0.5 * tij / yij;
                double fi1 = xx * Y1 * vol[j] / _den_i, fi2 = xx * Y2 * vol[j] / _den_i,
                       fi3 = xx * Y3 * vol[j] / _den_i;
                double fj1 = xx * Y1 * vol[i] / _den_j, fj2 = xx * Y2 * vol[i] / _den_j,
                       fj3 = xx * Y3 * vol[i] / _den_j;
                if (nthreads > 1) {
#pragma omp atomic
                    f[3 * i] += fi1;
#pragma omp atomic
                    f[3 * i + 1] += fi2;
#pragma omp atomic
                    f[3 * i + 2] += fi3;
#pragma omp atomic
                    f[3 * j] -= fj1;
#pragma omp atomic
                    f[3 * j + 1] -= fj2;
#pragma omp atomic
                    f[3 * j + 2] -= fj3;
                } else {
                    f[3 * i] = f[3 * i] + fi1;
                    f[3 * i + 1] = f[3 * i + 1] + fi2;
                    f[3 * i + 2] = f[3 * i + 2] + fi3;
                    f[3 * j] = f[3 * j] - fj1;
                    f[3 * j + 1] = f[3 * j + 1] - fj2;
                    f[3 * j + 2] = f[3 * j + 2] - fj3;
                }
            } else {
                COL(intact, M, k, i) = 0;
            }
        }
    }
}

/* Julia LinearAlgebra.norm (2-norm over all elements), summed in memory
 * order.  (The reference calls BLAS nrm2 for >= 32 elements, whose
 * internal order is library-specific; the gate below only differs from it
 * when d lies within a few ulps of the threshold.) */
static double norm2_seq(int64_t len, const double *a) {
    double s = 0.0;
    for (int64_t e = 0; e < len; ++e) s = s + a[e] * a[e];
    return sqrt(s);
}

/* general_material.jl:243-255 + Julia isapprox(x::AbstractArray, y) */
int or_isapprox_rigid(int64_t n, const double *y, const double *x) {
    const double rtol = 0x1p-26; /* sqrt(eps(Float64)) */
    int64_t len = 3 * n;
    double *A = (double *)malloc(sizeof(double) * (size_t)(len > 0 ? len : 1));
    double *D = (double *)malloc(sizeof(double) * (size_t)(len > 0 ? len : 1));
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            /* y_ .- y_[:, 1] .+ x[:, 1] */
            A[3 * i + d] = (y[3 * i + d] - y[d]) + x[d];
            D[3 * i + d] = A[3 * i + d] - x[3 * i + d];
        }
    double dn = norm2_seq(len, D);
    int res;
    if (isfinite(dn)) {
        double na = norm2_seq(len, A);
        double nx = norm2_seq(len, x);
        res = dn <= fmax(0.0, rtol * fmax(na, nx));
    } else {
        res = 1;
        for (int64_t e = 0; e < len; ++e) {
            double a = A[e], b = x[e];
            int ok = (a == b) || (isfinite(a) && isfinite(b) &&
                                  fabs(a - b) <= fmax(0.0, rtol * fmax(fabs(a), fabs(b))));
            if (!ok) {
                res = 0;
                break;
            }
        }
    }
    free(A);
    free(D);
    return res;
}

/* ------------------------------------------------------------------ */
/* Contacts                                                             */
/* ------------------------------------------------------------------ */

/* nonlinearspring.jl:124-145: returns 0 (scalar zero) or s .* dr */
static inline int contact_fn(double dr1, double dr2, double dr3, double equi_size,
                             double expo, double K, double *out) {
    double mag_dr = mag3(dr1, dr2, dr3);
    double del_x = equi_size - mag_dr;
    double strain = del_x / equi_size;
    if (del_x < 0.0) {
        out[0] = out[1] = out[2] = 0.0;
        return 0;
    }
    double s = (K * or_pow(strain, expo)) / (mag_dr + 1e-10);
    out[0] = s * dr1;
    out[1] = s * dr2;
    out[2] = s * dr3;
    return 1;
}

/* contacts.jl:403-416 collision_box + 434-476 update_contact_neighs! (12) */
void or_contact12_neighs(int64_t n1, const double *x11, int64_t n2,
                         const double *x22, double distance, int64_t rows,
                         int64_t *neighs) {
    memset(neighs, 0, sizeof(int64_t) * (size_t)rows * (size_t)n1);
    if (n1 == 0 || n2 == 0) return;
    double mn1[3], mx1[3], mn2[3], mx2[3], bmin[3], bmax[3];
    for (int d = 0; d < 3; ++d) {
        mn1[d] = mn2[d] = INFINITY;
        mx1[d] = mx2[d] = -INFINITY;
    }
    for (int64_t i = 0; i < n1; ++i)
        for (int d = 0; d < 3; ++d) {
            mn1[d] = fmin(mn1[d], x11[3 * i + d]);
            mx1[d] = fmax(mx1[d], x11[3 * i + d]);
        }
    for (int64_t i = 0; i < n2; ++i)
        for (int d = 0; d < 3; ++d) {
            mn2[d] = fmin(mn2[d], x22[3 * i + d]);
            mx2[d] = fmax(mx2[d], x22[3 * i + d]);
        }
    for (int d = 0; d < 3; ++d) {
        bmin[d] = fmax(mn1[d] - distance, mn2[d] - distance);
        bmax[d] = fmin(mx1[d] + distance, mx2[d] + distance);
    }
    double bvol = (bmax[0] - bmin[0]) * (bmax[1] - bmin[1]) * (bmax[2] - bmin[2]);
    if (bvol < 0.0) return; /* no overlap: neighs stay 0 */
    /* box members of pair[2], in ascending order (a_id) */
    int64_t *aid = (int64_t *)malloc(sizeof(int64_t) * (size_t)n2);
    int64_t nbox2 = 0;
    for (int64_t j = 0; j < n2; ++j) {
        int in = 1;
        for (int d = 0; d < 3; ++d) in &= (x22[3 * j + d] > bmin[d]) & (x22[3 * j + d] < bmax[d]);
        if (in) aid[nbox2++] = j;
    }
    const double dist2 = distance * distance;
    int64_t *cand = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nbox2 > 0 ? nbox2 : 1));
    for (int64_t i = 0; i < n1; ++i) {
        int in = 1;
        for (int d = 0; d < 3; ++d) in &= (x11[3 * i + d] > bmin[d]) & (x11[3 * i + d] < bmax[d]);
        if (!in) continue;
        double a1 = x11[3 * i], b1 = x11[3 * i + 1], c1 = x11[3 * i + 2];
        int64_t nc = 0;
        for (int64_t q = 0; q < nbox2; ++q) {
            int64_t j = aid[q];
            double a2 = x22[3 * j], b2 = x22[3 * j + 1], c2 = x22[3 * j + 2];
            if ((a1 - a2) * (a1 - a2) + (b1 - b2) * (b1 - b2) + (c1 - c2) * (c1 - c2) < dist2)
                cand[nc++] = j + 1; /* a_id is 1-based */
        }
        /* sort(family, dims=1) then rows end:-1:end+1-max_neighs:
         * the `rows` largest candidates, descending, zero padded */
        for (int64_t r = 0; r < rows && r < nc; ++r) COL(neighs, rows, r, i) = cand[nc - 1 - r];
    }
    free(cand);
    free(aid);
}

/* contacts.jl:210-247 short_range_contact! (12, CPU) */
void or_contact12_force(int64_t n1, int64_t rows, const int64_t *neighs,
                        const double *x1, const double *x2, double *f1,
                        double *f2, const double *vol1, const double *vol2,
                        const double *den1, const double *den2,
                        double equi_dist, double exponent, double stiffness) {
    double F[3];
    for (int64_t i = 0; i < n1; ++i) {
        double _den1_i = 1 / den1[i];
        for (int64_t k = 0; k < rows; ++k) {
            int64_t j = COL(neighs, rows, k, i);
            if (j > 0) {
                int64_t jj = j - 1;
                double _den2_j = 1 / den2[jj];
                double dr1 = x1[3 * i] - x2[3 * jj], dr2 = x1[3 * i + 1] - x2[3 * jj + 1],
                       dr3 = x1[3 * i + 2] - x2[3 * jj + 2];
                contact_fn(dr1, dr2, dr3, equi_dist, exponent, stiffness, F);
                double s1 = vol2[jj] * _den1_i, s2 = vol1[i] * _den2_j;
                for (int d = 0; d < 3; ++d) {
                    f1[3 * i + d] = f1[3 * i + d] + F[d] * s1;
                    f2[3 * jj + d] = f2[3 * jj + d] - F[d] * s2;
                }
            }
            if (j == 0) break;
        }
    }
}

/* peri.jl:500-520 get_cells + contacts.jl:539-573 (literal merge walk) and
 * the caller contacts.jl:591-605 (mask = any(family .> 0 .& .!intact)). */
void or_contact11_neighs(int64_t n, const double *x, int64_t M,
                         const int64_t *family, const uint8_t *intact,
                         double search_distance, double equi_dist,
                         int64_t max_part, int64_t rows, int64_t *neighbors) {
    memset(neighbors, 0, sizeof(int64_t) * (size_t)rows * (size_t)n);
    if (n == 0) return;
    int64_t *cell_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    cells_t c;
    get_cells(n, x, search_distance, max_part, &c, cell_of);
    const int64_t FS = M;
    const double equi_dist2 = equi_dist * equi_dist;
    int64_t nb[27];
    for (int64_t cell_i = 0; cell_i < c.ncells; ++cell_i) {
        int nn = neigh_cells(cell_i, c.N, nb);
        for (int64_t a = c.start[cell_i]; a < c.start[cell_i + 1]; ++a) {
            int64_t ca = c.idx[a];
            int64_t ind = 1;
            int mask = 0;
            for (int64_t k = 0; k < M; ++k)
                mask |= (COL(family, M, k, ca) > 0) & !COL(intact, M, k, ca);
            if (!mask) continue;
            double a1 = x[3 * ca], b1 = x[3 * ca + 1], c1 = x[3 * ca + 2];
            const int64_t *fms = family + (size_t)ca * (size_t)M;
            for (int q = 0; q < nn; ++q) {
                int64_t cell = nb[q];
                int64_t fm_ind = 1;
                for (int64_t b = c.start[cell]; b < c.start[cell + 1]; ++b) {
                    int64_t neigh = c.idx[b] + 1; /* 1-based, ascending */
                    while ((fms[fm_ind - 1] < neigh) && (fm_ind < FS)) fm_ind += 1;
                    if (fms[fm_ind - 1] == neigh) {
                        if (!COL(intact, M, fm_ind - 1, ca)) {
                            int64_t nj = neigh - 1;
                            double a2 = x[3 * nj], b2 = x[3 * nj + 1], c2 = x[3 * nj + 2];
                            double dr2 = ((a1 - a2) * (a1 - a2) + (b1 - b2) * (b1 - b2) + (c1 - c2) * (c1 - c2));
                            if (dr2 < equi_dist2) {
                                if (ind <= rows) COL(neighbors, rows, ind - 1, ca) = neigh;
                                ind += 1;
                            }
                        }
                    }
                }
            }
        }
    }
    free_cells(&c);
    free(cell_of);
}

/* Ordered variant of contacts.jl:539-573: what the merge walk there sets out
 * to find when families are not ascending.  Every family member j of a
 * particle i whose bond is broken, whose get_cells cell (peri.jl:500-520) is
 * one of the 27 around i's, and with |y_i - y_j|^2 < equi_dist^2 is listed,
 * in stored family order, up to rows; the rest of the column is 0. */
void or_contact11_neighs_ordered(int64_t n, const double *x, int64_t M,
                                 const int64_t *family, const uint8_t *intact,
                                 double search_distance, double equi_dist,
                                 int64_t max_part, int64_t rows, int64_t *neighbors) {
    memset(neighbors, 0, sizeof(int64_t) * (size_t)rows * (size_t)n);
    if (n == 0) return;
    int64_t *cell_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    cells_t c;
    get_cells(n, x, search_distance, max_part, &c, cell_of);
    const double equi_dist2 = equi_dist * equi_dist;
    const int64_t N0 = c.N[0], N1 = c.N[1];
    for (int64_t i = 0; i < n; ++i) {
        const int64_t ci = cell_of[i];
        const int64_t ii[3] = {ci % N0, (ci / N0) % N1, ci / (N0 * N1)};
        int64_t ind = 0;
        for (int64_t k = 0; k < M && ind < rows; ++k) {
            const int64_t j1 = COL(family, M, k, i);
            if (j1 <= 0 || COL(intact, M, k, i)) continue;
            const int64_t j = j1 - 1, cj = cell_of[j];
            const int64_t jj[3] = {cj % N0, (cj / N0) % N1, cj / (N0 * N1)};
            int adj = 1;
            for (int d = 0; d < 3; ++d) adj &= llabs(ii[d] - jj[d]) <= 1;
            const double d1 = x[3 * i] - x[3 * j], d2 = x[3 * i + 1] - x[3 * j + 1],
                         d3 = x[3 * i + 2] - x[3 * j + 2];
            const double dr2 = (d1 * d1 + d2 * d2) + d3 * d3;
            if (adj && dr2 < equi_dist2) COL(neighbors, rows, ind++, i) = j1;
        }
    }
    free_cells(&c);
    free(cell_of);
}

/* contacts.jl:357-381 short_range_contact! (11, CPU) */
void or_contact11_force(int64_t n, int64_t rows, const int64_t *neighs,
                        const double *x1, double *f1, const double *vol1,
                        const double *den1, double equi_dist, double exponent,
                        double stiffness) {
    double F[3];
    for (int64_t i = 0; i < n; ++i) {
        double _den_i = den1[i];
        for (int64_t k = 0; k < rows; ++k) {
            int64_t j = COL(neighs, rows, k, i);
            if (j != 0) {
                int64_t jj = j - 1;
                double _den_j = den1[jj];
                double dr1 = x1[3 * i] - x1[3 * jj], dr2 = x1[3 * i + 1] - x1[3 * jj + 1],
                       dr3 = x1[3 * i + 2] - x1[3 * jj + 2];
                contact_fn(dr1, dr2, dr3, equi_dist, exponent, stiffness, F);
                double si = vol1[jj] / _den_i, sj = vol1[jj] / _den_j;
                for (int d = 0; d < 3; ++d) {
                    f1[3 * i + d] = f1[3 * i + d] + F[d] * si;
                    f1[3 * jj + d] = f1[3 * jj + d] - F[d] * sj;
                }
            }
        }
    }
}

/* ---------------------------------------------------------------------
 * Elasto-plastic solid.  Both loops visit i = 1..n and the family of i in
 * stored order, like loop_over_neighs! (peri.jl:411-445) and
 * force_density_T! (general_material.jl:296-369).
 * --------------------------------------------------------------------- */
void or_td_norm2(int64_t n, int64_t M, const double *y, const double *x, const int64_t *family,
                 uint8_t *intact, const int64_t *type_rel, int64_t ntypes, const double *cs,
                 const double *vol, const double *m, const double *theta, const double *G,
                 const double *edp, double *td_norm2) {
    for (int64_t i = 0; i < n; ++i) td_norm2[i] = 0.0; /* elasto_plastic.jl:171 fill! */
    for (int64_t i = 0; i < n; ++i) {
        int64_t ti = type_rel[i];
        for (int64_t k = 0; k < M; ++k) {
            if (!COL(intact, M, k, i)) continue;
            int64_t j = COL(family, M, k, i) - 1;
            int64_t tj = type_rel[j];
            double X1 = x[3 * j] - x[3 * i], X2 = x[3 * j + 1] - x[3 * i + 1], X3 = x[3 * j + 2] - x[3 * i + 2];
            double Y1 = y[3 * j] - y[3 * i], Y2 = y[3 * j + 1] - y[3 * i + 1], Y3 = y[3 * j + 2] - y[3 * i + 2];
            double yij = mag3(Y1, Y2, Y3);
            double xij = mag3(X1, X2, X3);
            double extension = yij - xij;
            double s = extension / xij;
            size_t tp = (size_t)(ti - 1) + (size_t)(tj - 1) * (size_t)ntypes;
            if (s < cs[tp]) {
                /* elasto_plastic.jl:276-287 */
                double wij = 1 / mag3(X1, X2, X3);
                double wji = 1 / mag3(-X1, -X2, -X3);
                double Gij = G[tp];
                double edpij = COL(edp, M, k, i);
                double a = wij / m[i], b = wji / m[j];
                double w_m = a + b;
                double tw = theta[i] * a + theta[j] * b;
                double theta_ij = tw / w_m;
                double ed = extension - theta_ij * xij / 3;
                double td = 15 * Gij * (ed - edpij) * w_m;
                td_norm2[i] = td_norm2[i] + td * td * vol[j];
            } else {
                COL(intact, M, k, i) = 0;
            }
        }
    }
}

void or_force_density_ep(int64_t n, int64_t M, double *f, const double *y, const double *x,
                         const int64_t *family, uint8_t *intact, const int64_t *type_rel, int64_t ntypes,
                         const double *cs, const double *density, const double *vol, const double *m,
                         const double *theta, const double *K, const double *G, const double *psi,
                         const double *td_norm2, double *edp) {
    for (int64_t i = 0; i < n; ++i) {
        int64_t ti = type_rel[i];
        double _den_i = density[ti - 1];
        for (int64_t k = 0; k < M; ++k) {
            if (!COL(intact, M, k, i)) continue;
            int64_t j = COL(family, M, k, i) - 1;
            int64_t tj = type_rel[j];
            double _den_j = density[tj - 1];
            double X1 = x[3 * j] - x[3 * i], X2 = x[3 * j + 1] - x[3 * i + 1], X3 = x[3 * j + 2] - x[3 * i + 2];
            double Y1 = y[3 * j] - y[3 * i], Y2 = y[3 * j + 1] - y[3 * i + 1], Y3 = y[3 * j + 2] - y[3 * i + 2];
            double yij = mag3(Y1, Y2, Y3);
            double xij = mag3(X1, X2, X3);
            double extension = yij - xij;
            double s = extension / xij;
            size_t tp = (size_t)(ti - 1) + (size_t)(tj - 1) * (size_t)ntypes;
            if (s < cs[tp]) {
                /* elasto_plastic.jl:215-242 */
                double wij = 1 / mag3(X1, X2, X3);
                double wji = 1 / mag3(-X1, -X2, -X3);
                double Kij = K[tp], Gij = G[tp], psij = psi[tp];
                double C = sqrt(2 * psij / td_norm2[i]);
                double a = wij / m[i], b = wji / m[j];
                double tw = theta[i] * a + theta[j] * b;
                double theta_ij = tw / (a + b);
                double ed = extension - theta_ij * xij / 3;
                double ede = ed - COL(edp, M, k, i);
                double td_trial = 15 * Gij * (a + b) * ede;
                double td;
                if (C > 1) {
                    td = td_trial;
                } else {
                    td = C * td_trial;
                    COL(edp, M, k, i) = COL(edp, M, k, i) + ede * (1 - C);
                }
                double tn = (3 * Kij) * xij * tw;
                double tij = tn + td;
                double xx = 0.5 * tij / yij;
                f[3 * i] = f[3 * i] + xx * Y1 * vol[j] / _den_i;
                f[3 * i + 1] = f[3 * i + 1] + xx * Y2 * vol[j] / _den_i;
                f[3 * i + 2] = f[3 * i + 2] + xx * Y3 * vol[j] / _den_i;
                f[3 * j] = f[3 * j] - xx * Y1 * vol[i] / _den_j;
                f[3 * j + 1] = f[3 * j + 1] - xx * Y2 * vol[i] / _den_j;
                f[3 * j + 2] = f[3 * j + 2] - xx * Y3 * vol[i] / _den_j;
            } else {
                COL(intact, M, k, i) = 0;
            }
        }
    }
}
