// pd_contact.cu -- repulsive short-range contact (src/contacts/*.jl).
// Compiled with -fmad=false: forces must round like the reference CPU path.
//
// ContactModel12 (two blocks, pair[1] -> pair[2]):
//   neighbours (contacts.jl:434-476): for every pair[1] particle strictly
//   inside the collision box, the candidates are the pair[2] particles
//   strictly inside the box with d^2 < distance^2; the list keeps the
//   `rows` largest pair[2] indices in descending order.  Found here by a
//   cell list over the box (cells at least `distance` wide: complete).
//   forces (contacts.jl:210-247): pair[1] particle i adds F(i,j)*(V_j/rho_i)
//   over its list; pair[2] particle j subtracts F(i,j)*(V_i/rho_j) for every
//   i that lists it, in ascending i -- the serial loop's order, replayed as
//   a gather over a reverse list.
// ContactModel11 (self contact, contacts.jl:539-605 + 357-381): the
//   reference's merge walk compares the ascending cell members against the
//   family column from its top (the family is stored in descending order),
//   so the only member it can match is the column's first (largest) entry.
//   A particle therefore gets at most one contact neighbour: its first
//   family member q, when that bond is broken, q lies in one of the 27
//   reference cells around it (get_cells with max_part) and |y_i-y_q|^2 <
//   equi_dist^2.
#include <algorithm>
#include <cmath>
#include <vector>

#include "pd_env_impl.h"

using namespace pd;

namespace {

constexpr int kT = 256;
inline unsigned gridn(int64_t n, int t = kT) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

__device__ __forceinline__ double mag3(double a1, double a2, double a3) {
    return sqrt(a1 * a1 + a2 * a2 + a3 * a3);
}

// Julia pow_body (base/math.jl): compensated integer power; muladd fused.
__device__ double jl_pow_int(double x, long long n) {
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

__device__ double jl_pow(double x, double y) {
    if (x == 1.0) return 1.0;
    if (isnan(y)) return y;
    if (fabs(y) < 0x1.8p62) {
        long long yi = (long long)y;
        if ((double)yi == y) return yi == 0 ? 1.0 : jl_pow_int(x, yi);
    }
    return pow(x, y);
}

struct CLaw {
    double equi, expo, K;
};

// nonlinearspring.jl:133-143
__device__ __forceinline__ void contact_fn(const CLaw &c, double dr1, double dr2, double dr3, double &F1,
                                           double &F2, double &F3) {
    double mag_dr = mag3(dr1, dr2, dr3);
    double del_x = c.equi - mag_dr;
    double strain = del_x / c.equi;
    if (del_x < 0.0) {
        F1 = F2 = F3 = 0.0;
        return;
    }
    double s = (c.K * jl_pow(strain, c.expo)) / (mag_dr + 1e-10);
    F1 = s * dr1;
    F2 = s * dr2;
    F3 = s * dr3;
}

// Julia fld(x, y) for Float64: round((x - mod(x, y)) / y).
__device__ __forceinline__ double jl_fld(double x, double y) {
    double r;
    if (isinf(y) && isfinite(x)) r = x;
    else {
        r = fmod(x, y);
        if (r == 0.0) r = copysign(r, y);
        else if ((r > 0) != (y > 0)) r = r + y;
    }
    return rint((x - r) / y);
}

// ------------------------------- reductions ------------------------------
// Fixed partial-reduction width (blocks of the partial kernel, partials
// combined in block order): a constant rather than the device's SM count,
// so that the order of the reduction -- and its rounding -- does not depend
// on the GPU it runs on.
constexpr int kMMBlocks = 148;
__global__ void __launch_bounds__(kT)
    k_minmax_partial(int64_t first, int64_t n, const double4 *__restrict__ y, double *__restrict__ part) {
    __shared__ double sh[6][kT];
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = blockIdx.x * (int64_t)kT + threadIdx.x; i < n; i += (int64_t)kMMBlocks * kT) {
        double4 v = y[first + i];
        mn[0] = fmin(mn[0], v.x);
        mn[1] = fmin(mn[1], v.y);
        mn[2] = fmin(mn[2], v.z);
        mx[0] = fmax(mx[0], v.x);
        mx[1] = fmax(mx[1], v.y);
        mx[2] = fmax(mx[2], v.z);
    }
    for (int d = 0; d < 3; ++d) {
        sh[d][threadIdx.x] = mn[d];
        sh[3 + d][threadIdx.x] = mx[d];
    }
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int d = 0; d < 3; ++d) {
                sh[d][threadIdx.x] = fmin(sh[d][threadIdx.x], sh[d][threadIdx.x + s]);
                sh[3 + d][threadIdx.x] = fmax(sh[3 + d][threadIdx.x], sh[3 + d][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 6; ++d) part[6 * blockIdx.x + d] = sh[d][0];
}

__global__ void k_minmax_final(const double *__restrict__ part, double *__restrict__ out6) {
    double r[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int b = 0; b < kMMBlocks; ++b)
        for (int d = 0; d < 3; ++d) {
            r[d] = fmin(r[d], part[6 * b + d]);
            r[3 + d] = fmax(r[3 + d], part[6 * b + 3 + d]);
        }
    for (int d = 0; d < 6; ++d) out6[d] = r[d];
}

// ------------------------------- exclusive scan --------------------------
constexpr int kScanTile = 1024;
__global__ void __launch_bounds__(kScanTile)
    k_scan_tiles(int64_t n, const int32_t *__restrict__ in, int32_t *__restrict__ out, int32_t *__restrict__ sums) {
    __shared__ int32_t ws[32];
    int64_t i = blockIdx.x * (int64_t)kScanTile + threadIdx.x;
    int32_t v = i < n ? in[i] : 0, x = v;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        int32_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int32_t s = ws[lane], y = s;
        for (int o = 1; o < 32; o <<= 1) {
            int32_t t = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += t;
        }
        ws[lane] = y - s;
    }
    __syncthreads();
    int32_t incl = x + ws[w];
    if (i < n) out[i] = incl - v;
    if (threadIdx.x == kScanTile - 1) sums[blockIdx.x] = incl;
}

__global__ void k_scan_sums(int64_t ntiles, int32_t *__restrict__ sums) {
    // one thread, sequential: tile counts are small
    if (threadIdx.x != 0) return;
    int32_t run = 0;
    for (int64_t t = 0; t < ntiles; ++t) {
        int32_t s = sums[t];
        sums[t] = run;
        run += s;
    }
    sums[ntiles] = run;
}

__global__ void k_scan_add(int64_t n, int32_t *__restrict__ out, const int32_t *__restrict__ sums) {
    int64_t i = blockIdx.x * (int64_t)kScanTile + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

// out[0..n) = exclusive scan of in[0..n); returns the total via *total_dev
// (sums[ntiles]).  tmp needs ntiles+1 entries.
void scan_exclusive(cudaStream_t st, int64_t n, const int32_t *in, int32_t *out, int32_t *tmp) {
    int64_t nt = std::max<int64_t>(1, (n + kScanTile - 1) / kScanTile);
    k_scan_tiles<<<(unsigned)nt, kScanTile, 0, st>>>(n, in, out, tmp); pd::note_launch();
    k_scan_sums<<<1, 32, 0, st>>>(nt, tmp); pd::note_launch();
    k_scan_add<<<(unsigned)nt, kScanTile, 0, st>>>(n, out, tmp); pd::note_launch();
}

// ------------------------------- contact 12 ------------------------------
struct Box {
    double lo[3], hi[3];
    double inv_cell;
    int3 dims;
};

__device__ __forceinline__ bool in_box(const Box &b, double4 p) {
    return (p.x > b.lo[0]) & (p.x < b.hi[0]) & (p.y > b.lo[1]) & (p.y < b.hi[1]) & (p.z > b.lo[2]) &
           (p.z < b.hi[2]);
}

__device__ __forceinline__ int3 box_cell(const Box &b, double4 p) {
    int c[3];
    double v[3] = {p.x, p.y, p.z};
    for (int d = 0; d < 3; ++d) {
        double q = floor((v[d] - b.lo[d]) * b.inv_cell);
        int dm = d == 0 ? b.dims.x : (d == 1 ? b.dims.y : b.dims.z);
        if (!(q >= 0.0)) q = 0.0;
        if (q > dm - 1) q = dm - 1;
        c[d] = (int)q;
    }
    return make_int3(c[0], c[1], c[2]);
}

__global__ void k_c2_count(int64_t first2, int64_t n2, const double4 *__restrict__ y, Box b,
                           int32_t *__restrict__ cell_of, int32_t *__restrict__ ccount) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n2) return;
    double4 p = y[first2 + j];
    if (!in_box(b, p)) {
        cell_of[j] = -1;
        return;
    }
    int3 c = box_cell(b, p);
    int32_t id = c.x + b.dims.x * (c.y + b.dims.y * c.z);
    cell_of[j] = id;
    atomicAdd(&ccount[id], 1);
}

__global__ void k_c2_scatter(int64_t n2, const int32_t *__restrict__ cell_of, const int32_t *__restrict__ cstart,
                             int32_t *__restrict__ cursor, int32_t *__restrict__ clist) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n2) return;
    int32_t c = cell_of[j];
    if (c < 0) return;
    int32_t slot = atomicAdd(&cursor[c], 1);
    clist[cstart[c] + slot] = (int32_t)j;
}

template <bool kFill>
__global__ void k_c1_candidates(int64_t first1, int64_t n1, int64_t first2, const double4 *__restrict__ y, Box b,
                                double dist2, const int32_t *__restrict__ cstart, const int32_t *__restrict__ clist,
                                int32_t *__restrict__ ccount, const int32_t *__restrict__ coff,
                                int32_t *__restrict__ cand) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n1) return;
    double4 pi = y[first1 + i];
    int32_t k = 0;
    if (in_box(b, pi)) {
        int3 c = box_cell(b, pi);
        int32_t o = kFill ? coff[i] : 0;
        for (int dz = -1; dz <= 1; ++dz) {
            int z = c.z + dz;
            if (z < 0 || z >= b.dims.z) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                int yy = c.y + dy;
                if (yy < 0 || yy >= b.dims.y) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    int x = c.x + dx;
                    if (x < 0 || x >= b.dims.x) continue;
                    int32_t cell = x + b.dims.x * (yy + b.dims.y * z);
                    for (int32_t s = cstart[cell]; s < cstart[cell + 1]; ++s) {
                        int32_t j = clist[s];
                        double4 pj = y[first2 + j];
                        double a = pi.x - pj.x, bb = pi.y - pj.y, cc = pi.z - pj.z;
                        if (a * a + bb * bb + cc * cc < dist2) {
                            if (kFill) cand[o + k] = j;
                            ++k;
                        }
                    }
                }
            }
        }
    }
    if (!kFill) ccount[i] = k;
}

// sort candidates descending and keep the `rows` largest (column-major nb).
__global__ void k_c1_select(int64_t n1, int64_t rows, int64_t first2, const int32_t *__restrict__ coff,
                            int32_t *__restrict__ cand, int32_t *__restrict__ nb) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n1) return;
    int32_t o = coff[i], n = coff[i + 1] - o;
    int32_t *a = cand + o;
    for (int32_t k = 1; k < n; ++k) {
        int32_t v = a[k], j = k - 1;
        while (j >= 0 && a[j] < v) {
            a[j + 1] = a[j];
            --j;
        }
        a[j + 1] = v;
    }
    for (int64_t r = 0; r < rows; ++r) nb[r * n1 + i] = r < n ? (int32_t)(first2 + a[r]) : -1;
}

// reverse lists: for set-2 particle j, the set-1 particles listing it.
__global__ void k_rev_count(int64_t n1, int64_t rows, int64_t first2, const int32_t *__restrict__ nb,
                            int32_t *__restrict__ rcnt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n1) return;
    for (int64_t r = 0; r < rows; ++r) {
        int32_t j = nb[r * n1 + i];
        if (j < 0) break;
        atomicAdd(&rcnt[j - first2], 1);
    }
}

__global__ void k_rev_fill(int64_t n1, int64_t rows, int64_t first1, int64_t first2, const int32_t *__restrict__ nb,
                           const int32_t *__restrict__ roff, int32_t *__restrict__ cursor, int32_t *__restrict__ rev) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n1) return;
    for (int64_t r = 0; r < rows; ++r) {
        int32_t j = nb[r * n1 + i];
        if (j < 0) break;
        int32_t s = atomicAdd(&cursor[j - first2], 1);
        rev[roff[j - first2] + s] = (int32_t)(first1 + i);
    }
}

__global__ void k_rev_sort(int64_t n2, const int32_t *__restrict__ roff, int32_t *__restrict__ rev) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n2) return;
    int32_t o = roff[j], n = roff[j + 1] - o;
    int32_t *a = rev + o;
    for (int32_t k = 1; k < n; ++k) {
        int32_t v = a[k], m = k - 1;
        while (m >= 0 && a[m] > v) {
            a[m + 1] = a[m];
            --m;
        }
        a[m + 1] = v;
    }
}

// contacts.jl:230-245, pair[1] side: f_i += F .* (V_j * (1/rho_i))
__global__ void k_c12_force1(int64_t first1, int64_t n1, int64_t rows, const int32_t *__restrict__ nb,
                             const double4 *__restrict__ y, const double4 *__restrict__ x4,
                             const double *__restrict__ dens, CLaw law, double4 *__restrict__ f) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n1) return;
    int64_t p = first1 + i;
    double4 yi = y[p], fi = f[p];
    double inv_den1 = 1 / dens[p];
    for (int64_t r = 0; r < rows; ++r) {
        int32_t j = nb[r * n1 + i];
        if (j < 0) break;
        double4 yj = y[j];
        double F1, F2, F3;
        contact_fn(law, yi.x - yj.x, yi.y - yj.y, yi.z - yj.z, F1, F2, F3);
        double s = x4[j].w * inv_den1;
        fi.x = fi.x + F1 * s;
        fi.y = fi.y + F2 * s;
        fi.z = fi.z + F3 * s;
    }
    f[p] = fi;
}

// pair[2] side: f_j -= F(i,j) .* (V_i * (1/rho_j)) for i ascending
__global__ void k_c12_force2(int64_t first2, int64_t n2, const int32_t *__restrict__ roff,
                             const int32_t *__restrict__ rev, const double4 *__restrict__ y,
                             const double4 *__restrict__ x4, const double *__restrict__ dens, CLaw law,
                             double4 *__restrict__ f) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n2) return;
    int32_t o = roff[j], e = roff[j + 1];
    if (o == e) return;
    int64_t q = first2 + j;
    double4 yj = y[q], fj = f[q];
    double inv_den2 = 1 / dens[q];
    for (int32_t r = o; r < e; ++r) {
        int32_t i = rev[r];
        double4 yi = y[i];
        double F1, F2, F3;
        contact_fn(law, yi.x - yj.x, yi.y - yj.y, yi.z - yj.z, F1, F2, F3);
        double s = x4[i].w * inv_den2;
        fj.x = fj.x - F1 * s;
        fj.y = fj.y - F2 * s;
        fj.z = fj.z - F3 * s;
    }
    f[q] = fj;
}

// ------------------------------- contact 11 ------------------------------
struct RefCells {
    double mn[3];
    double h;
    double maxpart;
};

__device__ __forceinline__ int ref_cell(const RefCells &c, double v, int d) {
    double q = jl_fld(v - c.mn[d], c.h);
    return (int)fmax(1.0, fmin(c.maxpart, q));
}

__global__ void k_c11_neighs(int64_t first, int64_t n, const double4 *__restrict__ y,
                             const SliceInfo *__restrict__ si, const int32_t *__restrict__ cnt,
                             const int32_t *__restrict__ nbr, const uint32_t *__restrict__ words,
                             const uint32_t *__restrict__ fam, RefCells rc, double equi2,
                             int32_t *__restrict__ nb11) {
    int64_t li = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (li >= n) return;
    int64_t p = first + li;
    int32_t res = -1;
    // The first family member is the first slot whose family bit is set.
    const BondRef fr = bond_ref(si, nbr, fam, p);
    const int32_t c = cnt[p];
    int32_t k0 = -1;
    for (int32_t k = 0; k < c; k += 32) {
        uint32_t m = *fr.word(k);
        if (m) {
            k0 = k + __ffs(m) - 1;
            break;
        }
    }
    if (k0 >= 0) {
        const uint32_t w = words[(fr.w - fam) + 32 * (int64_t)(k0 >> 5)];
        bool intact0 = (w >> (k0 & 31)) & 1u;
        if (!intact0) {
            int32_t q = fr.q(k0);
            double4 a = y[p], b = y[q];
            bool adj = abs(ref_cell(rc, a.x, 0) - ref_cell(rc, b.x, 0)) <= 1 &&
                       abs(ref_cell(rc, a.y, 1) - ref_cell(rc, b.y, 1)) <= 1 &&
                       abs(ref_cell(rc, a.z, 2) - ref_cell(rc, b.z, 2)) <= 1;
            double d1 = a.x - b.x, d2 = a.y - b.y, d3 = a.z - b.z;
            double dr2 = d1 * d1 + d2 * d2 + d3 * d3;
            if (adj && dr2 < equi2) res = q;
        }
    }
    nb11[li] = res;
}

// Every family member with a broken bond, in an adjacent search cell and
// within equi_dist, in family (slot) order, up to rows.
__global__ void k_c11_neighs_ordered(int64_t first, int64_t n, const double4 *__restrict__ y,
                                     const SliceInfo *__restrict__ si, const int32_t *__restrict__ cnt,
                                     const int32_t *__restrict__ nbr, const uint32_t *__restrict__ words,
                                     const uint32_t *__restrict__ fam, RefCells rc, double equi2, int64_t rows,
                                     int32_t *__restrict__ nb) {
    int64_t li = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (li >= n) return;
    int64_t p = first + li;
    const BondRef fr = bond_ref(si, nbr, fam, p);
    const int64_t wb = fr.w - fam;
    const int32_t c = cnt[p];
    const double4 a = y[p];
    int64_t r = 0;
    for (int32_t k = 0; k < c && r < rows; ++k) {
        const uint32_t bit = 1u << (k & 31);
        const int64_t wi = wb + 32 * (int64_t)(k >> 5);
        if (!(fam[wi] & bit) || (words[wi] & bit)) continue;  // not a member, or intact
        const int32_t q = fr.q(k);
        const double4 b = y[q];
        const bool adj = abs(ref_cell(rc, a.x, 0) - ref_cell(rc, b.x, 0)) <= 1 &&
                         abs(ref_cell(rc, a.y, 1) - ref_cell(rc, b.y, 1)) <= 1 &&
                         abs(ref_cell(rc, a.z, 2) - ref_cell(rc, b.z, 2)) <= 1;
        const double d1 = a.x - b.x, d2 = a.y - b.y, d3 = a.z - b.z;
        const double dr2 = ((d1 * d1 + d2 * d2) + d3 * d3);
        if (adj && dr2 < equi2) nb[r++ * n + li] = q;
    }
    for (; r < rows; ++r) nb[r * n + li] = -1;
}

__global__ void k_c11_rev_count(int64_t first, int64_t n, const int32_t *__restrict__ nb11, int32_t *__restrict__ rcnt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t q = nb11[i];
    if (q >= 0) atomicAdd(&rcnt[q - first], 1);
}

__global__ void k_c11_rev_fill(int64_t first, int64_t n, const int32_t *__restrict__ nb11,
                               const int32_t *__restrict__ roff, int32_t *__restrict__ cursor,
                               int32_t *__restrict__ rev) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t q = nb11[i];
    if (q < 0) return;
    int32_t s = atomicAdd(&cursor[q - first], 1);
    rev[roff[q - first] + s] = (int32_t)(first + i);
}

// contacts.jl:366-379 in serial order for particle p:
//   i < p listing p:  f_p -= F(y_i - y_p) .* (V_p / rho_p)
//   own neighbour q:  f_p += F(y_p - y_q) .* (V_q / rho_p)
//   i > p listing p:  f_p -= F(y_i - y_p) .* (V_p / rho_p)
__global__ void k_c11_force(int64_t first, int64_t n, int64_t nbrows, const int32_t *__restrict__ nb11,
                            const int32_t *__restrict__ roff, const int32_t *__restrict__ rev,
                            const double4 *__restrict__ y, const double4 *__restrict__ x4,
                            const double *__restrict__ dens, CLaw law, double4 *__restrict__ f) {
    int64_t li = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (li >= n) return;
    int64_t p = first + li;
    int32_t o = roff[li], e = roff[li + 1];
    if (o == e && nb11[li] < 0) return;
    double4 yp = y[p], fp = f[p];
    double den_p = dens[p], vol_p = x4[p].w;
    double F1, F2, F3;
    int32_t r = o;
    for (; r < e && rev[r] < p; ++r) {
        double4 yi = y[rev[r]];
        contact_fn(law, yi.x - yp.x, yi.y - yp.y, yi.z - yp.z, F1, F2, F3);
        double s = vol_p / den_p;
        fp.x = fp.x - F1 * s;
        fp.y = fp.y - F2 * s;
        fp.z = fp.z - F3 * s;
    }
    for (int64_t k = 0; k < nbrows; ++k) {  // p's own neighbours, in row order
        const int32_t q = nb11[k * n + li];
        if (q < 0) break;
        double4 yq = y[q];
        contact_fn(law, yp.x - yq.x, yp.y - yq.y, yp.z - yq.z, F1, F2, F3);
        double s = x4[q].w / den_p;
        fp.x = fp.x + F1 * s;
        fp.y = fp.y + F2 * s;
        fp.z = fp.z + F3 * s;
    }
    for (; r < e; ++r) {
        double4 yi = y[rev[r]];
        contact_fn(law, yi.x - yp.x, yi.y - yp.y, yi.z - yp.z, F1, F2, F3);
        double s = vol_p / den_p;
        fp.x = fp.x - F1 * s;
        fp.y = fp.y - F2 * s;
        fp.z = fp.z - F3 * s;
    }
    f[p] = fp;
}

pd_status minmax(pd_env *env, int64_t first, int64_t n, double *out6_host) {
    if (!env->red.p || env->red.n < 6 * kMMBlocks + 6) PD_TRY(env->red.alloc(6 * kMMBlocks + 6 + 512));
    k_minmax_partial<<<kMMBlocks, kT, 0, env->st>>>(first, n, env->y.p, env->red.p); pd::note_launch();
    k_minmax_final<<<1, 1, 0, env->st>>>(env->red.p, env->red.p + 6 * kMMBlocks); pd::note_launch();
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out6_host, env->red.p + 6 * kMMBlocks, 6 * sizeof(double), cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

pd_status build_reverse(pd_env *env, DevContact &dc, int64_t n_src, int64_t src_first, int64_t n_tgt,
                        int64_t tgt_first, const int32_t *nb, int64_t rows, bool c11) {
    cudaStream_t st = env->st;
    CK(cudaMemsetAsync(dc.rev_cnt.p, 0, (n_tgt + 1) * 4, st));
    if (c11) k_c11_rev_count<<<gridn(n_src), kT, 0, st>>>(src_first, n_src, nb, dc.rev_cnt.p);
    else k_rev_count<<<gridn(n_src), kT, 0, st>>>(n_src, rows, tgt_first, nb, dc.rev_cnt.p);
    pd::note_launch();
    PD_TRY(grow(dc.s_rtmp, (n_tgt + 1 + kScanTile - 1) / kScanTile + 2));
    scan_exclusive(st, n_tgt + 1, dc.rev_cnt.p, dc.rev_off.p, dc.s_rtmp.p);
    int32_t total = 0;
    CK(cudaMemcpyAsync(&total, dc.rev_off.p + n_tgt, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (total > dc.rev_cap) {
        PD_TRY(dc.rev.alloc(total + 1024));
        dc.rev_cap = total + 1024;
    }
    CK(cudaMemsetAsync(dc.rev_cnt.p, 0, (n_tgt + 1) * 4, st));
    if (c11) k_c11_rev_fill<<<gridn(n_src), kT, 0, st>>>(src_first, n_src, nb, dc.rev_off.p, dc.rev_cnt.p, dc.rev.p);
    else k_rev_fill<<<gridn(n_src), kT, 0, st>>>(n_src, rows, src_first, tgt_first, nb, dc.rev_off.p, dc.rev_cnt.p,
                                                 dc.rev.p);
    pd::note_launch();
    k_rev_sort<<<gridn(n_tgt), kT, 0, st>>>(n_tgt, dc.rev_off.p, dc.rev.p); pd::note_launch();
    CK(cudaGetLastError());
    return PD_OK;
}

// Lists of the particles with contact work (local indices; order free: each
// particle's own sum does not depend on it).
__global__ void k_active(int64_t n_src, const int32_t *__restrict__ nb, int64_t n_tgt,
                         const int32_t *__restrict__ roff, int self, int32_t *__restrict__ act1,
                         int32_t *__restrict__ act2, int32_t *__restrict__ counts) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n_src && (nb[i] >= 0 || (self && roff[i + 1] > roff[i]))) act1[atomicAdd(&counts[0], 1)] = (int32_t)i;
    if (!self && i < n_tgt && roff[i + 1] > roff[i]) act2[atomicAdd(&counts[1], 1)] = (int32_t)i;
}

pd_status build_active(pd_env *env, DevContact &dc, bool self) {
    cudaStream_t st = env->st;
    const int64_t n2 = self ? dc.n1 : dc.n2;
    if ((int64_t)dc.act1.n < dc.n1) PD_TRY(dc.act1.alloc(std::max<int64_t>(dc.n1, 1)));
    if (!self && (int64_t)dc.act2.n < n2) PD_TRY(dc.act2.alloc(std::max<int64_t>(n2, 1)));
    if (!dc.act_n.p) PD_TRY(dc.act_n.alloc(2));
    CK(cudaMemsetAsync(dc.act_n.p, 0, 2 * sizeof(int32_t), st));
    const int64_t n = std::max(dc.n1, n2);
    k_active<<<gridn(n), kT, 0, st>>>(dc.n1, dc.nb.p, n2, dc.rev_off.p, self ? 1 : 0, dc.act1.p,
                                      self ? nullptr : dc.act2.p, dc.act_n.p);
    pd::note_launch();
    int32_t h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, dc.act_n.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    dc.nact1 = h[0];
    dc.nact2 = self ? 0 : h[1];
    return PD_OK;
}

pd_status update12(pd_env *env, const HostContact &hc, DevContact &dc) {
    cudaStream_t st = env->st;
    const int64_t n1 = dc.n1, n2 = dc.n2;
    CK(cudaMemsetAsync(dc.nb.p, 0xff, (size_t)n1 * dc.rows * 4, st));
    double m1[6], m2[6];
    PD_TRY(minmax(env, dc.first1, n1, m1));
    PD_TRY(minmax(env, dc.first2, n2, m2));
    // contacts.jl:403-416 collision_box
    const double skin = hc.distance;
    Box b;
    for (int d = 0; d < 3; ++d) {
        b.lo[d] = std::max(m1[d] - skin, m2[d] - skin);
        b.hi[d] = std::min(m1[3 + d] + skin, m2[3 + d] + skin);
    }
    double bvol = (b.hi[0] - b.lo[0]) * (b.hi[1] - b.lo[1]) * (b.hi[2] - b.lo[2]);
    dc.has_neighs = true;
    if (bvol < 0.0) {
        PD_TRY(build_reverse(env, dc, n1, dc.first1, n2, dc.first2, dc.nb.p, dc.rows, false));
        return build_active(env, dc, false);
    }
    double cell = hc.distance * (1.0 + 1e-9);
    int dims[3];
    double tot = 1.0;
    for (int d = 0; d < 3; ++d) {
        double nd = std::floor(std::max(0.0, b.hi[d] - b.lo[d]) / cell) + 1.0;
        nd = std::min(nd, 512.0);
        dims[d] = (int)nd;
        tot *= nd;
    }
    // keep the grid bounded: coarser cells are still complete
    while (tot > 16.0e6) {
        for (int d = 0; d < 3; ++d) dims[d] = std::max(1, dims[d] / 2);
        tot = (double)dims[0] * dims[1] * dims[2];
    }
    double width = 0.0;
    for (int d = 0; d < 3; ++d) width = std::max(width, (b.hi[d] - b.lo[d]) / dims[d]);
    b.inv_cell = 1.0 / std::max(width * (1.0 + 1e-9), cell);
    b.dims = make_int3(dims[0], dims[1], dims[2]);
    const int64_t ncell = (int64_t)dims[0] * dims[1] * dims[2];
    DBuf<int32_t> &cell_of = dc.s_cell_of, &ccount = dc.s_ccount, &cstart = dc.s_cstart, &cursor = dc.s_cursor,
                  &clist = dc.s_clist, &tmp = dc.s_tmp, &c1cnt = dc.s_c1cnt, &c1off = dc.s_c1off, &cand = dc.s_cand;
    PD_TRY(grow(cell_of, n2));
    PD_TRY(grow(ccount, ncell + 1));
    PD_TRY(grow(cstart, ncell + 1));
    PD_TRY(grow(cursor, ncell + 1));
    PD_TRY(grow(clist, n2));
    PD_TRY(grow(tmp, (std::max(ncell, n1) + 1 + kScanTile - 1) / kScanTile + 2));
    CK(cudaMemsetAsync(ccount.p, 0, (ncell + 1) * 4, st));
    CK(cudaMemsetAsync(cursor.p, 0, (ncell + 1) * 4, st));
    k_c2_count<<<gridn(n2), kT, 0, st>>>(dc.first2, n2, env->y.p, b, cell_of.p, ccount.p); pd::note_launch();
    scan_exclusive(st, ncell + 1, ccount.p, cstart.p, tmp.p);
    k_c2_scatter<<<gridn(n2), kT, 0, st>>>(n2, cell_of.p, cstart.p, cursor.p, clist.p); pd::note_launch();
    const double dist2 = hc.distance * hc.distance;
    PD_TRY(grow(c1cnt, n1 + 1));
    PD_TRY(grow(c1off, n1 + 1));
    CK(cudaMemsetAsync(c1cnt.p, 0, (n1 + 1) * 4, st));
    k_c1_candidates<false><<<gridn(n1), kT, 0, st>>>(dc.first1, n1, dc.first2, env->y.p, b, dist2, cstart.p, clist.p,
                                                     c1cnt.p, nullptr, nullptr); pd::note_launch();
    scan_exclusive(st, n1 + 1, c1cnt.p, c1off.p, tmp.p);
    int32_t total = 0;
    CK(cudaMemcpyAsync(&total, c1off.p + n1, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    PD_TRY(grow(cand, std::max<int32_t>(total, 1)));
    k_c1_candidates<true><<<gridn(n1), kT, 0, st>>>(dc.first1, n1, dc.first2, env->y.p, b, dist2, cstart.p, clist.p,
                                                    nullptr, c1off.p, cand.p); pd::note_launch();
    k_c1_select<<<gridn(n1), kT, 0, st>>>(n1, dc.rows, dc.first2, c1off.p, cand.p, dc.nb.p); pd::note_launch();
    CK(cudaGetLastError());
    PD_TRY(build_reverse(env, dc, n1, dc.first1, n2, dc.first2, dc.nb.p, dc.rows, false));
    return build_active(env, dc, false);
}

pd_status update11(pd_env *env, const HostContact &hc, DevContact &dc, int64_t max_part) {
    cudaStream_t st = env->st;
    double m[6];
    PD_TRY(minmax(env, dc.first1, dc.n1, m));
    RefCells rc;
    for (int d = 0; d < 3; ++d) rc.mn[d] = m[d];
    rc.h = hc.distance;
    rc.maxpart = (double)max_part;
    if (hc.kind == PD_CONTACT_11_ORDERED) {
        k_c11_neighs_ordered<<<gridn(dc.n1), kT, 0, st>>>(dc.first1, dc.n1, env->y.p, env->sinfo.p, env->cnt.p,
                                                          env->nbr.p, env->words[env->cur].p, env->fam.p, rc,
                                                          hc.equi_dist * hc.equi_dist, dc.nbrows, dc.nb.p);
        pd::note_launch();
    } else {
        k_c11_neighs<<<gridn(dc.n1), kT, 0, st>>>(dc.first1, dc.n1, env->y.p, env->sinfo.p, env->cnt.p, env->nbr.p,
                                                  env->words[env->cur].p, env->fam.p, rc, hc.equi_dist * hc.equi_dist,
                                                  dc.nb.p);
        pd::note_launch();
    }
    CK(cudaGetLastError());
    dc.has_neighs = true;
    PD_TRY(build_reverse(env, dc, dc.n1, dc.first1, dc.n1, dc.first1, dc.nb.p, dc.nbrows,
                         hc.kind != PD_CONTACT_11_ORDERED));
    return build_active(env, dc, true);
}

}  // namespace

namespace pd {

pd_status contacts_finalize(pd_env *env) {
    for (auto &hc : env->hc) {
        DevContact dc;
        const HostBlock &b1 = env->hb[hc.b1], &b2 = env->hb[hc.b2];
        // The reference selects contact particles by type range
        // (contacts.jl:212-219); with disjoint block type ranges this is the
        // block itself.
        for (size_t k = 0; k < env->hb.size(); ++k) {
            const HostBlock &o = env->hb[k];
            for (int64_t blk : {hc.b1, hc.b2}) {
                if ((int64_t)k == blk) continue;
                const HostBlock &t = env->hb[blk];
                bool overlap = o.type_start < t.type_start + t.nt && t.type_start < o.type_start + o.nt;
                if (overlap)
                    return fail(PD_ERR_UNSUPPORTED,
                                "contact model needs block type ranges that no other block shares");
            }
        }
        dc.n1 = b1.n;
        dc.first1 = b1.first_int;
        if (hc.kind == PD_CONTACT_12) {
            dc.n2 = b2.n;
            dc.first2 = b2.first_int;
            dc.rows = std::min<int64_t>(hc.max_neighs, b2.n);  // ContactModel12_gcal
            dc.nbrows = dc.rows;
            PD_TRY(dc.nb.alloc((size_t)dc.n1 * dc.rows));
            CK(cudaMemsetAsync(dc.nb.p, 0xff, (size_t)dc.n1 * dc.rows * 4, env->st));
            PD_TRY(dc.rev_off.alloc(dc.n2 + 1));
            PD_TRY(dc.rev_cnt.alloc(dc.n2 + 1));
            CK(cudaMemsetAsync(dc.rev_off.p, 0, (dc.n2 + 1) * 4, env->st));
        } else {
            dc.n2 = b1.n;
            dc.first2 = b1.first_int;
            dc.rows = hc.max_neighs;  // ContactModel11_gcal: zeros(max_neighs, N)
            dc.nbrows = hc.kind == PD_CONTACT_11_ORDERED ? dc.rows : 1;
            PD_TRY(dc.nb.alloc((size_t)dc.n1 * dc.nbrows));
            CK(cudaMemsetAsync(dc.nb.p, 0xff, (size_t)dc.n1 * dc.nbrows * 4, env->st));
            PD_TRY(dc.rev_off.alloc(dc.n1 + 1));
            PD_TRY(dc.rev_cnt.alloc(dc.n1 + 1));
            CK(cudaMemsetAsync(dc.rev_off.p, 0, (dc.n1 + 1) * 4, env->st));
        }
        PD_TRY(dc.rev.alloc(1024));
        dc.rev_cap = 1024;
        hc.rows = dc.rows;
        env->contacts.push_back(std::move(dc));
    }
    return PD_OK;
}

pd_status contacts_update_neighs(pd_env *env, int64_t max_part) {
    ++env->contact_epoch;  // captured contact steps of older lists are stale
    for (size_t k = 0; k < env->hc.size(); ++k) {
        if (env->hc[k].kind == PD_CONTACT_12) PD_TRY(update12(env, env->hc[k], env->contacts[k]));
        else PD_TRY(update11(env, env->hc[k], env->contacts[k], max_part));
    }
    return PD_OK;
}

pd_status contacts_force(pd_env *env) {
    for (size_t k = 0; k < env->hc.size(); ++k) {
        const HostContact &hc = env->hc[k];
        DevContact &dc = env->contacts[k];
        if (!dc.has_neighs) continue;  // neighbour lists start empty (zeros)
        CLaw law{hc.equi_dist, hc.exponent, hc.stiffness};
        if (hc.kind == PD_CONTACT_12) {
            k_c12_force1<<<gridn(dc.n1), kT, 0, env->st>>>(dc.first1, dc.n1, dc.rows, dc.nb.p, env->y.p, env->x4.p,
                                                           env->dens.p, law, env->f.p); pd::note_launch();
            k_c12_force2<<<gridn(dc.n2), kT, 0, env->st>>>(dc.first2, dc.n2, dc.rev_off.p, dc.rev.p, env->y.p,
                                                           env->x4.p, env->dens.p, law, env->f.p); pd::note_launch();
        } else {
            k_c11_force<<<gridn(dc.n1), kT, 0, env->st>>>(dc.first1, dc.n1, dc.nbrows, dc.nb.p, dc.rev_off.p, dc.rev.p, env->y.p,
                                                          env->x4.p, env->dens.p, law, env->f.p); pd::note_launch();
        }
        CK(cudaGetLastError());
    }
    return PD_OK;
}

}  // namespace pd

extern "C" pd_status pd_env_get_contact_neighs(pd_env *env, int64_t contact, int64_t *rows, int64_t *neighs) {
    if (!env) return fail(PD_ERR_ARG, "environment handle is NULL");
    if (!env->finalized) return fail(PD_ERR_STATE, "environment is not finalized");
    if (contact < 0 || contact >= (int64_t)env->hc.size() || !rows) return fail(PD_ERR_ARG, "bad contact or NULL rows");
    const HostContact &hc = env->hc[contact];
    DevContact &dc = env->contacts[contact];
    *rows = dc.rows;
    if (!neighs) return PD_OK;
    CK(cudaSetDevice(env->device));
    std::fill(neighs, neighs + (size_t)dc.rows * dc.n1, 0);
    if (hc.kind == PD_CONTACT_12) {
        std::vector<int32_t> h((size_t)dc.n1 * dc.rows);
        CK(cudaMemcpyAsync(h.data(), dc.nb.p, h.size() * 4, cudaMemcpyDeviceToHost, env->st));
        CK(cudaStreamSynchronize(env->st));
        for (int64_t i = 0; i < dc.n1; ++i)
            for (int64_t r = 0; r < dc.rows; ++r) {
                int32_t j = h[r * dc.n1 + i];
                neighs[(size_t)i * dc.rows + r] = j < 0 ? 0 : (int64_t)(j - dc.first2 + 1);
            }
    } else {
        std::vector<int32_t> h((size_t)dc.n1 * dc.nbrows);
        CK(cudaMemcpyAsync(h.data(), dc.nb.p, h.size() * 4, cudaMemcpyDeviceToHost, env->st));
        CK(cudaStreamSynchronize(env->st));
        for (int64_t i = 0; i < dc.n1; ++i)
            for (int64_t r = 0; r < dc.nbrows; ++r) {
                const int32_t j = h[r * dc.n1 + i];
                neighs[(size_t)i * dc.rows + r] = j < 0 ? 0 : (int64_t)(j - dc.first1 + 1);
            }
    }
    return PD_OK;
}
