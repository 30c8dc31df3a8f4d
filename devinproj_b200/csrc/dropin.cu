// FP64 drop-in kernels: cell grid, full neighbour list, LJ and DSF forces, VelocityVerlet, reductions.
//
// These back the reference-shaped plug-ins (LennardJones / DampedShiftedCoulomb / VelocityVerlet) when
// called one force evaluation at a time. Arithmetic follows the reference's FP64 NumPy expressions
// (accusim/forces.py:119-175, :279-321, :408-452; accusim/integrators.py:25-31); the pair filter and
// the integrator use non-contracted IEEE operations so their decisions and updates are bit-identical.
#include <math.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"

using namespace acs;

namespace {

struct GridDev {
  double lo[3], span[3];
  Box3 box;
  int nc[3];
  double rc2;
};

GridDev to_dev(const acs_grid* g) {
  GridDev d;
  for (int k = 0; k < 3; ++k) {
    d.lo[k] = g->lo[k];
    d.span[k] = g->span[k];
    d.box.L[k] = g->box[k];
    d.box.inv[k] = g->box[k] != 0.0 ? 1.0 / g->box[k] : 0.0;
    d.nc[k] = g->ncell[k];
  }
  d.box.periodic = g->periodic;
  d.rc2 = g->rc2;
  return d;
}

// cell = clip(int((pos - lo) / span * ncell), 0, ncell - 1)   (accusim/forces.py:290-291)
__device__ __forceinline__ int bin1(double x, double lo, double span, int nc) {
  double t = mul(div(sub(x, lo), span), (double)nc);
  if (!(t >= 1.0)) return 0;  // also catches NaN
  if (t >= (double)(nc - 1)) return nc - 1;
  return (int)t;
}

__global__ void k_bin(const double* __restrict__ pos, int64_t n, GridDev g, int32_t* __restrict__ cell_of,
                      int32_t* __restrict__ count) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c0 = bin1(pos[3 * i + 0], g.lo[0], g.span[0], g.nc[0]);
  int c1 = bin1(pos[3 * i + 1], g.lo[1], g.span[1], g.nc[1]);
  int c2 = bin1(pos[3 * i + 2], g.lo[2], g.span[2], g.nc[2]);
  int c = (c0 * g.nc[1] + c1) * g.nc[2] + c2;
  cell_of[i] = c;
  atomicAdd(&count[c], 1);
}

// Three-phase exclusive scan over int32 (chunk of 4096 per 1024-thread block).
constexpr int kScanThreads = 1024, kScanPer = 4, kScanChunk = kScanThreads * kScanPer;

__device__ int block_exclusive_scan(int v, int* total) {
  __shared__ int warp_sums[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_sums[lane] = w;
  }
  __syncthreads();
  int excl = x - v + (wid > 0 ? warp_sums[wid - 1] : 0);
  if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return excl;
}

__global__ void k_scan_chunks(const int32_t* __restrict__ in, int32_t* __restrict__ out, int64_t len,
                              int32_t* __restrict__ chunk_sums) {
  int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanPer;
  int v[kScanPer];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = (base + k < len) ? in[base + k] : 0;
    s += v[k];
  }
  int total;
  int e = block_exclusive_scan(s, &total);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < len) out[base + k] = e;
    e += v[k];
  }
  if (threadIdx.x == 0) chunk_sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(int32_t* __restrict__ sums, int64_t nchunks, int32_t* __restrict__ grand_total) {
  // one block; serial over groups of 1024 chunk sums with a running carry
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b = 0; b < nchunks; b += blockDim.x) {
    int64_t idx = b + threadIdx.x;
    int v = idx < nchunks ? sums[idx] : 0;
    int total;
    int e = block_exclusive_scan(v, &total);
    if (idx < nchunks) sums[idx] = e + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0 && grand_total) *grand_total = carry;
}

__global__ void k_scan_add(int32_t* __restrict__ out, int64_t len, const int32_t* __restrict__ sums) {
  int64_t base = (int64_t)blockIdx.x * kScanChunk;
  int add_v = sums[blockIdx.x];
  for (int k = threadIdx.x; k < kScanChunk; k += blockDim.x)
    if (base + k < len) out[base + k] += add_v;
}

__global__ void k_scatter(const int32_t* __restrict__ cell_of, int64_t n, const int32_t* __restrict__ start,
                          int32_t* __restrict__ cursor, int32_t* __restrict__ cell_atoms) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = cell_of[i];
  int slot = atomicAdd(&cursor[c], 1);
  cell_atoms[start[c] + slot] = (int32_t)i;
}

// Atoms of a cell in ascending index order, so list order is deterministic run to run: every atom's rank among
// its cell's atoms (the scatter's arbitrary order in `unsorted`) gives its place. A thread per atom; the reads
// of a cell's members are shared by the cell's atoms through L1.
__global__ void k_rank_cells(const int32_t* __restrict__ cell_of, int64_t n, const int32_t* __restrict__ start,
                             const int32_t* __restrict__ unsorted, int32_t* __restrict__ cell_atoms) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cell_of[i];
  const int s = start[c], e = start[c + 1];
  int rank = 0;
  for (int b = s; b < e; ++b) rank += unsorted[b] < (int32_t)i;
  cell_atoms[s + rank] = (int32_t)i;
}

__device__ __forceinline__ void stencil_range(int c, int nc, int periodic, int& lo, int& hi) {
  if (periodic) {
    if (nc >= 3) { lo = -1; hi = 1; } else { lo = 0; hi = 0; }
  } else {
    lo = (c > 0) ? -1 : 0;
    hi = (c < nc - 1) ? 1 : 0;
  }
}

__device__ __forceinline__ int wrap_cell(int c, int nc) { return c < 0 ? c + nc : (c >= nc ? c - nc : c); }

__global__ void k_list(const double* __restrict__ pos, int64_t n, GridDev g, const int32_t* __restrict__ cell_of,
                       const int32_t* __restrict__ start, const int32_t* __restrict__ cell_atoms, int maxnb,
                       int32_t* __restrict__ nbr, int32_t* __restrict__ nnb, acs_dev_status* status) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cell_of[i];
  const int c2 = c % g.nc[2], c1 = (c / g.nc[2]) % g.nc[1], c0 = c / (g.nc[2] * g.nc[1]);
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
  int lo0, hi0, lo1, hi1, lo2, hi2;
  stencil_range(c0, g.nc[0], g.box.periodic, lo0, hi0);
  stencil_range(c1, g.nc[1], g.box.periodic, lo1, hi1);
  stencil_range(c2, g.nc[2], g.box.periodic, lo2, hi2);
  int cnt = 0;
  for (int a = lo0; a <= hi0; ++a) {
    const int n0 = wrap_cell(c0 + a, g.nc[0]);
    for (int b = lo1; b <= hi1; ++b) {
      const int n1 = wrap_cell(c1 + b, g.nc[1]);
      for (int d = lo2; d <= hi2; ++d) {
        const int n2 = wrap_cell(c2 + d, g.nc[2]);
        const int nb = (n0 * g.nc[1] + n1) * g.nc[2] + n2;
        for (int k = start[nb], e = start[nb + 1]; k < e; ++k) {
          const int j = cell_atoms[k];
          if (j == i) continue;
          double dx = sub(pos[3 * (int64_t)j], xi), dy = sub(pos[3 * (int64_t)j + 1], yi),
                 dz = sub(pos[3 * (int64_t)j + 2], zi);
          min_image3(dx, dy, dz, g.box);
          if (norm2(dx, dy, dz) < g.rc2) {
            if (cnt < maxnb) nbr[nbr_slot(i, cnt, maxnb)] = j;
            ++cnt;
          }
        }
      }
    }
  }
  nnb[i] = cnt;
  if (cnt > maxnb) {
    atomicOr(&status->flags, ACS_FLAG_OVERFLOW);
    atomicMax(&status->need_nbr, cnt);
  }
}

// Pair-distance histogram of accusim/analysis.py:7-24 (rdf): pairs i < j, both of `species` (all when < 0),
// minimum-image r by the reference's FP64 expression, binned by NumPy's uniform-bin rule on [0, rmax]
// (numpy histogram: index = int((r / rmax) * bins), the right edge into the last bin, then one step down if
// r < edge[index] or up if r >= edge[index + 1] below the last bin, with edge[k] = k * (rmax / bins) and
// edge[bins] = rmax). Per-block shared-memory counts, integer atomics: exact and order-independent.
__global__ void k_rdf(const double* __restrict__ pos, const int32_t* __restrict__ sp, int64_t n, GridDev g,
                      const int32_t* __restrict__ cell_of, const int32_t* __restrict__ start,
                      const int32_t* __restrict__ cell_atoms, int species, int bins, double rmax, double step,
                      unsigned long long* __restrict__ hist) {
  extern __shared__ unsigned int sh_hist[];
  for (int b = threadIdx.x; b < bins; b += blockDim.x) sh_hist[b] = 0u;
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && (species < 0 || sp[i] == species)) {
    const int c = cell_of[i];
    const int c2 = c % g.nc[2], c1 = (c / g.nc[2]) % g.nc[1], c0 = c / (g.nc[2] * g.nc[1]);
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    int lo0, hi0, lo1, hi1, lo2, hi2;
    stencil_range(c0, g.nc[0], g.box.periodic, lo0, hi0);
    stencil_range(c1, g.nc[1], g.box.periodic, lo1, hi1);
    stencil_range(c2, g.nc[2], g.box.periodic, lo2, hi2);
    for (int a = lo0; a <= hi0; ++a) {
      const int n0 = wrap_cell(c0 + a, g.nc[0]);
      for (int b = lo1; b <= hi1; ++b) {
        const int n1 = wrap_cell(c1 + b, g.nc[1]);
        for (int d = lo2; d <= hi2; ++d) {
          const int n2 = wrap_cell(c2 + d, g.nc[2]);
          const int nb = (n0 * g.nc[1] + n1) * g.nc[2] + n2;
          for (int k = start[nb], e = start[nb + 1]; k < e; ++k) {
            const int j = cell_atoms[k];
            if (j <= i || (species >= 0 && sp[j] != species)) continue;
            double dx = sub(pos[3 * (int64_t)j], xi), dy = sub(pos[3 * (int64_t)j + 1], yi),
                   dz = sub(pos[3 * (int64_t)j + 2], zi);
            min_image3(dx, dy, dz, g.box);
            const double r = __dsqrt_rn(norm2(dx, dy, dz));
            if (!(r <= rmax)) continue;
            int idx = (int)mul(__ddiv_rn(r, rmax), (double)bins);
            if (idx == bins) idx -= 1;
            if (r < mul((double)idx, step)) idx -= 1;
            const double upper = idx + 1 == bins ? rmax : mul((double)(idx + 1), step);
            if (r >= upper && idx != bins - 1) idx += 1;
            atomicAdd(&sh_hist[idx], 1u);
          }
        }
      }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < bins; b += blockDim.x)
    if (sh_hist[b]) atomicAdd(&hist[b], (unsigned long long)sh_hist[b]);
}

__global__ void k_pairs(const int32_t* __restrict__ nbr, const int32_t* __restrict__ nnb, int64_t n, int maxnb,
                        int32_t* pi, int32_t* pj, int64_t cap, unsigned long long* count) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int m = min(nnb[i], maxnb);
  for (int k = 0; k < m; ++k) {
    int j = nbr[nbr_slot(i, k, maxnb)];
    if (i < j) {
      unsigned long long w = atomicAdd(count, 1ull);
      if ((int64_t)w < cap) {
        pi[w] = (int32_t)i;
        pj[w] = j;
      }
    }
  }
}

__global__ void k_displacement(const double* __restrict__ pos, const double* __restrict__ pos0, int64_t n, Box3 box,
                               double half_skin2, int32_t* flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dx = sub(pos[3 * i], pos0[3 * i]), dy = sub(pos[3 * i + 1], pos0[3 * i + 1]),
         dz = sub(pos[3 * i + 2], pos0[3 * i + 2]);
  min_image3(dx, dy, dz, box);
  if (!(norm2(dx, dy, dz) < half_skin2)) *flag = 1;  // NaN also forces a rebuild, as in the reference
}

// ------------------------------------------------------------------------------------ forces --
struct LJTab {
  int ns;
  double eps[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  double sig2[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  double rc2[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  double shift6;  // src6**2 - src6, src6 = (1/cutoff**2)**3
};

struct DSFPar {
  double a, rc, k, c, erc, fshift, self_coef;
};

template <bool DENSE>
__global__ void __launch_bounds__(kBlock) k_lj64(const double* __restrict__ pos, const int32_t* __restrict__ sp, int64_t n,
                                                  Box3 box, const int32_t* __restrict__ nbr,
                                                  const int32_t* __restrict__ nnb, int maxnb, LJTab t,
                                                  double* __restrict__ force, double* partials, unsigned int* ticket,
                                                  double* energy) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double fx = 0.0, fy = 0.0, fz = 0.0, u = 0.0;
  if (i < n) {
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    const int si = sp[i] * t.ns;
    const int64_t m = DENSE ? n : (int64_t)min(nnb[i], maxnb);
    for (int64_t k = 0; k < m; ++k) {
      const int64_t j = DENSE ? k : (int64_t)nbr[nbr_slot(i, (int)k, maxnb)];
      if (DENSE && j == i) continue;
      double dx = sub(pos[3 * j], xi), dy = sub(pos[3 * j + 1], yi), dz = sub(pos[3 * j + 2], zi);
      min_image3(dx, dy, dz, box);
      const double r2 = norm2(dx, dy, dz);
      const int p = si + sp[j];
      const double e = t.eps[p];
      if (r2 < t.rc2[p] && e > 0.0) {
        const double ir2 = 1.0 / r2;
        const double sr2 = t.sig2[p] * ir2;
        const double sr6 = sr2 * sr2 * sr2;
        u += 4.0 * e * (sr6 * sr6 - sr6 - t.shift6);
        const double coef = -24.0 * e * (2.0 * sr6 * sr6 - sr6) * ir2;
        fx += coef * dx;
        fy += coef * dy;
        fz += coef * dz;
      }
    }
    force[3 * i] = fx;
    force[3 * i + 1] = fy;
    force[3 * i + 2] = fz;
  }
  double v[1] = {0.5 * u};
  block_sum_finish<1>(v, partials, ticket, energy);
}

template <bool DENSE>
__global__ void __launch_bounds__(kBlock) k_dsf64(const double* __restrict__ pos, const double* __restrict__ q, int64_t n,
                                                   Box3 box, const int32_t* __restrict__ nbr,
                                                   const int32_t* __restrict__ nnb, int maxnb,
                                                   const int32_t* __restrict__ ex_start,
                                                   const int32_t* __restrict__ ex_idx, DSFPar P,
                                                   double* __restrict__ force, double* partials, unsigned int* ticket,
                                                   double* energy) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double fx = 0.0, fy = 0.0, fz = 0.0, u = 0.0;
  if (i < n) {
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2], qi = q[i];
    const int xs = ex_start ? ex_start[i] : 0, xe = ex_start ? ex_start[i + 1] : 0;
    const int64_t m = DENSE ? n : (int64_t)min(nnb[i], maxnb);
    for (int64_t k = 0; k < m; ++k) {
      const int64_t j = DENSE ? k : (int64_t)nbr[nbr_slot(i, (int)k, maxnb)];
      if (DENSE && j == i) continue;
      double dx = sub(pos[3 * j], xi), dy = sub(pos[3 * j + 1], yi), dz = sub(pos[3 * j + 2], zi);
      min_image3(dx, dy, dz, box);
      const double r = sqrt(norm2(dx, dy, dz));
      if (!(r < P.rc)) continue;
      bool excluded = false;
      for (int x = xs; x < xe; ++x) excluded |= (ex_idx[x] == (int32_t)j);
      if (excluded) continue;
      const double qq = qi * q[j];
      const double ar = P.a * r;
      const double er = erfc(ar);
      const double ir = 1.0 / r;
      u += qq * (er * ir - P.erc / P.rc + P.fshift * (r - P.rc));
      const double fv = qq * ((er * (ir * ir) + P.c * exp(-(ar * ar)) * ir) - P.fshift) * ir;
      fx -= fv * dx;
      fy -= fv * dy;
      fz -= fv * dz;
    }
    force[3 * i] = P.k * fx;
    force[3 * i + 1] = P.k * fy;
    force[3 * i + 2] = P.k * fz;
    u = P.k * (0.5 * u - qi * qi * P.self_coef);
  }
  double v[1] = {u};
  block_sum_finish<1>(v, partials, ticket, energy);
}

// ------------------------------------------------------------------------------- integrator --
__global__ void k_kick(double* __restrict__ vel, const double* __restrict__ acc, int64_t n3, double h) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) vel[i] = add(vel[i], mul(h, acc[i]));  // vel += (0.5*dt) * acc
}

// pos %= box with NumPy's remainder: r = fmod(x, L); r += L if r and L differ in sign.
__device__ __forceinline__ double py_mod(double x, double L) {
  double r = fmod(x, L);
  if (r != 0.0) {
    if ((L < 0.0) != (r < 0.0)) r = add(r, L);
  } else {
    r = copysign(0.0, L);
  }
  return r;
}

__global__ void k_drift_wrap(double* __restrict__ pos, const double* __restrict__ vel, int64_t n, double dt, Box3 box) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double x = add(pos[3 * i + d], mul(dt, vel[3 * i + d]));
    if (box.periodic) x = py_mod(x, box.L[d]);
    pos[3 * i + d] = x;
  }
}

// Langevin O-step: vel = c1 * vel + sig[atom] * noise (accusim/integrators.py:66-67, no FMA).
__global__ void k_langevin_ou(double* __restrict__ vel, const double* __restrict__ noise,
                              const double* __restrict__ sig, int64_t n3, double c1) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) vel[i] = add(mul(c1, vel[i]), mul(sig[i / 3], noise[i]));
}

struct MassTab {
  double m[ACS_MAX_SPECIES];
};

__global__ void k_accel(double* __restrict__ acc, const double* __restrict__ force, const int32_t* __restrict__ sp,
                        MassTab mt, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double m = mt.m[sp[i]];
#pragma unroll
  for (int d = 0; d < 3; ++d) acc[3 * i + d] = div(force[3 * i + d], m);
}

__global__ void __launch_bounds__(kBlock) k_conserved(const double* __restrict__ pos, const double* __restrict__ vel,
                                                       const int32_t* __restrict__ sp, MassTab mt, int64_t n,
                                                       double* partials, unsigned int* ticket, double* out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  if (i < n) {
    const double m = mt.m[sp[i]];
    const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    const double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
    v[0] = 0.5 * (m * (vx * vx) + m * (vy * vy) + m * (vz * vz));
    const double px = m * vx, py = m * vy, pz = m * vz;
    v[1] = px;
    v[2] = py;
    v[3] = pz;
    v[4] = y * pz - z * py;
    v[5] = z * px - x * pz;
    v[6] = x * py - y * px;
  }
  block_sum_finish<7>(v, partials, ticket, out);
}

inline Box3 make_box(const double* box3, int periodic) {
  Box3 b;
  for (int k = 0; k < 3; ++k) {
    b.L[k] = box3 ? box3[k] : 0.0;
    b.inv[k] = b.L[k] != 0.0 ? 1.0 / b.L[k] : 0.0;
  }
  b.periodic = (periodic && box3) ? 1 : 0;
  return b;
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

inline int64_t grid_cells(const acs_grid* g) { return (int64_t)g->ncell[0] * g->ncell[1] * g->ncell[2]; }

// CPython float floor division (Objects/floatobject.c float_divmod), as used by `span // rc`.
double py_floordiv(double a, double b) {
  double mod = fmod(a, b);
  double dv = (a - mod) / b;
  if (mod != 0.0) {
    if ((b < 0) != (mod < 0)) dv -= 1.0;
  }
  double fl;
  if (dv != 0.0) {
    fl = floor(dv);
    if (dv - fl > 0.5) fl += 1.0;
  } else {
    fl = copysign(0.0, a / b);
  }
  return fl;
}

constexpr int kRdfMaxBins = 8192;   // shared-memory counts per block

// Cell binning shared by the list build and the pair histogram: atoms counted into cells, exclusive scan,
// scatter, deterministic in-cell order (ascending atom index).
struct CellBins {
  int32_t *cell_of, *start, *cell_atoms;
};
int bin_cells(const double* pos, int64_t n, const acs_grid* g, void* work, cudaStream_t s, CellBins& cb) {
  const int64_t nc = grid_cells(g);
  const int64_t nchunks = ceil_div(nc + 1, kScanChunk);
  char* w = (char*)work;
  cb.cell_of = (int32_t*)w; w += align256(n * 4);
  int32_t* count = (int32_t*)w; w += align256((nc + 1) * 4);
  cb.start = (int32_t*)w; w += align256((nc + 1) * 4);
  cb.cell_atoms = (int32_t*)w; w += align256(n * 4);
  int32_t* unsorted = (int32_t*)w; w += align256(n * 4);
  int32_t* sums = (int32_t*)w;
  GridDev gd = to_dev(g);
  if (cudaMemsetAsync(count, 0, (nc + 1) * 4, s) != cudaSuccess) return 1;
  const int nb = (int)ceil_div(n, kBlock);
  k_bin<<<nb, kBlock, 0, s>>>(pos, n, gd, cb.cell_of, count);
  k_scan_chunks<<<(int)nchunks, kScanThreads, 0, s>>>(count, cb.start, nc + 1, sums);
  k_scan_sums<<<1, kScanThreads, 0, s>>>(sums, nchunks, nullptr);
  k_scan_add<<<(int)nchunks, 256, 0, s>>>(cb.start, nc + 1, sums);
  if (cudaMemsetAsync(count, 0, (nc + 1) * 4, s) != cudaSuccess) return 1;
  k_scatter<<<nb, kBlock, 0, s>>>(cb.cell_of, n, cb.start, count, unsorted);
  k_rank_cells<<<nb, kBlock, 0, s>>>(cb.cell_of, n, cb.start, unsorted, cb.cell_atoms);
  return 0;
}

}  // namespace

// ===================================================================================== C ABI ==
extern "C" {

int acs_abi_version(void) { return ACS_ABI_VERSION; }

const char* acs_status_string(int s) {
  switch (s) {
    case ACS_OK: return "ok";
    case ACS_ERR_ARG: return "bad argument";
    case ACS_ERR_WORKSPACE: return "workspace too small";
    case ACS_ERR_CUDA: return "CUDA runtime error";
    case ACS_ERR_LIST_OVERFLOW: return "neighbour list capacity exceeded";
    case ACS_ERR_NONFINITE: return "non-finite force or position";
    case ACS_ERR_TIMEOUT: return "device barrier wait timed out";
    case ACS_ERR_UNSUPPORTED: return "unsupported size or mode";
    case ACS_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

int acs_device_info(int* sm_count, int* cc_major, int* cc_minor) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ACS_ERR_NO_DEVICE;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return ACS_ERR_NO_DEVICE;
  if (sm_count) *sm_count = p.multiProcessorCount;
  if (cc_major) *cc_major = p.major;
  if (cc_minor) *cc_minor = p.minor;
  return ACS_OK;
}

int acs_grid_setup(acs_grid* g, const double* box3, int periodic, const double* lo3, const double* hi3, double rc) {
  if (!g || !(rc > 0.0) || (!box3 && (!lo3 || !hi3))) return ACS_ERR_ARG;
  for (int k = 0; k < 3; ++k) {
    double lo, span;
    if (box3) {
      lo = 0.0;
      span = box3[k];
    } else {
      lo = lo3[k];
      span = std::max(hi3[k] - lo, rc);
    }
    if (!(span > 0.0)) return ACS_ERR_ARG;
    double nc = std::max(py_floordiv(span, rc), 1.0);
    if (nc > 2097152.0) return ACS_ERR_UNSUPPORTED;
    int ic = (int)nc;
    if (periodic && box3 && ic < 3) ic = 1;
    g->lo[k] = lo;
    g->span[k] = span;
    g->box[k] = box3 ? box3[k] : 0.0;
    g->ncell[k] = ic;
  }
  if (grid_cells(g) > (int64_t)INT32_MAX / 2) return ACS_ERR_UNSUPPORTED;
  g->periodic = (periodic && box3) ? 1 : 0;
  g->rc = rc;
  g->rc2 = rc * rc;
  return ACS_OK;
}

size_t acs_nlist_work_bytes(int64_t n, const acs_grid* g) {
  if (!g || n < 0) return 0;
  const int64_t nc = grid_cells(g);
  const int64_t nchunks = ceil_div(nc + 1, kScanChunk);
  return align256(n * 4) + 2 * align256((nc + 1) * 4) + 2 * align256(n * 4) + align256((nchunks + 1) * 4);
}

int acs_nlist_build(const double* pos, int64_t n, const acs_grid* g, int32_t maxnb, int32_t* nbr, int32_t* nnb,
                    void* work, size_t work_bytes, acs_dev_status* status, void* stream) {
  if (!g || n < 0 || maxnb < 1 || n > INT32_MAX || (n > 0 && (!pos || !nbr || !nnb || !work || !status)))
    return ACS_ERR_ARG;
  if (work_bytes < acs_nlist_work_bytes(n, g)) return ACS_ERR_WORKSPACE;
  if (n == 0) return ACS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nc = grid_cells(g);
  const int64_t nchunks = ceil_div(nc + 1, kScanChunk);
  CellBins cb;
  if (bin_cells(pos, n, g, work, s, cb)) return ACS_ERR_CUDA;
  k_list<<<(int)ceil_div(n, kBlock), kBlock, 0, s>>>(pos, n, to_dev(g), cb.cell_of, cb.start, cb.cell_atoms, maxnb,
                                                     nbr, nnb, status);
  return launch_status();
}

size_t acs_rdf_work_bytes(int64_t n, const acs_grid* g) { return acs_nlist_work_bytes(n, g); }

int acs_rdf_hist(const double* pos, const int32_t* sp, int64_t n, const acs_grid* g, int32_t species, int32_t bins,
                 double rmax, unsigned long long* hist, void* work, size_t work_bytes, void* stream) {
  if (!g || n < 0 || n > INT32_MAX || bins < 1 || bins > kRdfMaxBins || !(rmax > 0.0) || !hist ||
      (n > 0 && (!pos || !work || (species >= 0 && !sp))))
    return ACS_ERR_ARG;
  if (!g->periodic || !(g->rc >= rmax)) return ACS_ERR_ARG;   // cells no narrower than rmax, periodic box
  if (work_bytes < acs_rdf_work_bytes(n, g)) return ACS_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * bins, s) != cudaSuccess) return ACS_ERR_CUDA;
  if (n == 0) return ACS_OK;
  CellBins cb;
  if (bin_cells(pos, n, g, work, s, cb)) return ACS_ERR_CUDA;
  k_rdf<<<(int)ceil_div(n, kBlock), kBlock, sizeof(unsigned int) * bins, s>>>(
      pos, sp, n, to_dev(g), cb.cell_of, cb.start, cb.cell_atoms, species, bins, rmax, rmax / bins, hist);
  return launch_status();
}

int acs_nlist_pairs(const int32_t* nbr, const int32_t* nnb, int64_t n, int32_t maxnb, int32_t* pi, int32_t* pj,
                    int64_t cap, unsigned long long* count_dev, void* stream) {
  if (n < 0 || maxnb < 1 || !count_dev || (n > 0 && (!nbr || !nnb)) || (cap > 0 && (!pi || !pj))) return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(count_dev, 0, sizeof(unsigned long long), s) != cudaSuccess) return ACS_ERR_CUDA;
  if (n == 0) return ACS_OK;
  k_pairs<<<(int)ceil_div(n, kBlock), kBlock, 0, s>>>(nbr, nnb, n, maxnb, pi, pj, cap, count_dev);
  return launch_status();
}

int acs_nlist_displacement(const double* pos, const double* pos0, int64_t n, const double* box3, int periodic,
                           double half_skin2, int32_t* flag_dev, void* stream) {
  if (n < 0 || !flag_dev || (n > 0 && (!pos || !pos0))) return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(flag_dev, 0, 4, s) != cudaSuccess) return ACS_ERR_CUDA;
  if (n == 0) return ACS_OK;
  k_displacement<<<(int)ceil_div(n, kBlock), kBlock, 0, s>>>(pos, pos0, n, make_box(box3, periodic), half_skin2,
                                                              flag_dev);
  return launch_status();
}

size_t acs_force_work_bytes(int64_t n) { return align256(std::max<int64_t>(ceil_div(n, kBlock), 1) * 8) + 256; }

static int reduce_setup(void* work, size_t work_bytes, size_t need, int64_t nblocks, int width, double** partials,
                        unsigned int** ticket, cudaStream_t s) {
  if (work_bytes < need) return ACS_ERR_WORKSPACE;
  *partials = (double*)work;
  *ticket = (unsigned int*)((char*)work + align256(nblocks * width * 8));
  return cudaMemsetAsync(*ticket, 0, 4, s) == cudaSuccess ? ACS_OK : ACS_ERR_CUDA;
}

int acs_lj_fp64(const double* pos, const int32_t* sp, int64_t n, const double* box3, int periodic,
                const int32_t* nbr, const int32_t* nnb, int32_t maxnb, int32_t n_species, const double* eps_tab,
                const double* sig_tab, double cutoff, double* force, double* energy_dev, void* work,
                size_t work_bytes, void* stream) {
  if (n < 1 || n > INT32_MAX || !pos || !sp || !force || !energy_dev || !eps_tab || !sig_tab || n_species < 1 ||
      n_species > ACS_MAX_SPECIES || !(cutoff > 0.0) || (nbr && (!nnb || maxnb < 1)))
    return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nb = ceil_div(n, kBlock);
  double* partials;
  unsigned int* ticket;
  int st = reduce_setup(work, work_bytes, acs_force_work_bytes(n), nb, 1, &partials, &ticket, s);
  if (st) return st;
  LJTab t;
  t.ns = n_species;
  for (int a = 0; a < n_species * n_species; ++a) {
    t.eps[a] = eps_tab[a];
    t.sig2[a] = sig_tab[a] * sig_tab[a];                       // sig ** 2
    const double rc = cutoff * sig_tab[a];
    t.rc2[a] = rc * rc;                                        // (cutoff * sig) ** 2
  }
  const double c2 = cutoff * cutoff;
  const double src6 = (1.0 / c2) * (1.0 / c2) * (1.0 / c2);
  t.shift6 = src6 * src6 - src6;
  Box3 b = make_box(box3, periodic);
  if (nbr)
    k_lj64<false><<<(int)nb, kBlock, 0, s>>>(pos, sp, n, b, nbr, nnb, maxnb, t, force, partials, ticket, energy_dev);
  else
    k_lj64<true><<<(int)nb, kBlock, 0, s>>>(pos, sp, n, b, nullptr, nullptr, 0, t, force, partials, ticket,
                                           energy_dev);
  return launch_status();
}

int acs_dsf_fp64(const double* pos, const double* q, int64_t n, const double* box3, int periodic,
                 const int32_t* nbr, const int32_t* nnb, int32_t maxnb, const int32_t* ex_start,
                 const int32_t* ex_idx, double alpha, double rcut, double k, double* force, double* energy_dev,
                 void* work, size_t work_bytes, void* stream) {
  if (n < 1 || n > INT32_MAX || !pos || !q || !force || !energy_dev || !(rcut > 0.0) || !(alpha >= 0.0) ||
      (nbr && (!nnb || maxnb < 1)) || (ex_start && !ex_idx))
    return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nb = ceil_div(n, kBlock);
  double* partials;
  unsigned int* ticket;
  int st = reduce_setup(work, work_bytes, acs_force_work_bytes(n), nb, 1, &partials, &ticket, s);
  if (st) return st;
  DSFPar P;
  P.a = alpha;
  P.rc = rcut;
  P.k = k;
  P.c = 2.0 * alpha / sqrt(M_PI);
  P.erc = erfc(alpha * rcut);
  P.fshift = P.erc / (rcut * rcut) + P.c * exp(-((alpha * rcut) * (alpha * rcut))) / rcut;
  P.self_coef = P.erc / (2.0 * rcut) + alpha / sqrt(M_PI);
  Box3 b = make_box(box3, periodic);
  if (nbr)
    k_dsf64<false><<<(int)nb, kBlock, 0, s>>>(pos, q, n, b, nbr, nnb, maxnb, ex_start, ex_idx, P, force, partials,
                                             ticket, energy_dev);
  else
    k_dsf64<true><<<(int)nb, kBlock, 0, s>>>(pos, q, n, b, nullptr, nullptr, 0, ex_start, ex_idx, P, force,
                                            partials, ticket, energy_dev);
  return launch_status();
}

int acs_vv_kick(double* vel, const double* acc, int64_t n, double half_dt, void* stream) {
  if (n < 0 || (n > 0 && (!vel || !acc))) return ACS_ERR_ARG;
  if (n == 0) return ACS_OK;
  k_kick<<<(int)ceil_div(3 * n, kBlock), kBlock, 0, (cudaStream_t)stream>>>(vel, acc, 3 * n, half_dt);
  return launch_status();
}

int acs_vv_drift_wrap(double* pos, const double* vel, int64_t n, double dt, const double* box3, int periodic,
                      void* stream) {
  if (n < 0 || (n > 0 && (!pos || !vel))) return ACS_ERR_ARG;
  if (n == 0) return ACS_OK;
  k_drift_wrap<<<(int)ceil_div(n, kBlock), kBlock, 0, (cudaStream_t)stream>>>(pos, vel, n, dt,
                                                                                make_box(box3, periodic));
  return launch_status();
}

int acs_langevin_ou(double* vel, const double* noise, const double* sig, int64_t n, double c1, void* stream) {
  if (n < 0 || (n > 0 && (!vel || !noise || !sig))) return ACS_ERR_ARG;
  if (n == 0) return ACS_OK;
  k_langevin_ou<<<(int)ceil_div(3 * n, kBlock), kBlock, 0, (cudaStream_t)stream>>>(vel, noise, sig, 3 * n, c1);
  return launch_status();
}

int acs_vv_accel(double* acc, const double* force, const int32_t* sp, const double* species_mass, int32_t n_species,
                 int64_t n, void* stream) {
  if (n < 0 || (n > 0 && (!acc || !force || !sp || !species_mass)) || n_species < 1 || n_species > ACS_MAX_SPECIES)
    return ACS_ERR_ARG;
  if (n == 0) return ACS_OK;
  MassTab mt;
  for (int a = 0; a < ACS_MAX_SPECIES; ++a) mt.m[a] = a < n_species ? species_mass[a] : 1.0;
  k_accel<<<(int)ceil_div(n, kBlock), kBlock, 0, (cudaStream_t)stream>>>(acc, force, sp, mt, n);
  return launch_status();
}

size_t acs_reduce_work_bytes(int64_t n) { return align256(std::max<int64_t>(ceil_div(n, kBlock), 1) * 7 * 8) + 256; }

int acs_reduce_conserved(const double* pos, const double* vel, const int32_t* sp, const double* species_mass,
                         int32_t n_species, int64_t n, double* out_dev, void* work, size_t work_bytes, void* stream) {
  if (n < 1 || !pos || !vel || !sp || !species_mass || !out_dev || n_species < 1 || n_species > ACS_MAX_SPECIES)
    return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nb = ceil_div(n, kBlock);
  double* partials;
  unsigned int* ticket;
  int st = reduce_setup(work, work_bytes, acs_reduce_work_bytes(n), nb, 7, &partials, &ticket, s);
  if (st) return st;
  MassTab mt;
  for (int a = 0; a < ACS_MAX_SPECIES; ++a) mt.m[a] = a < n_species ? species_mass[a] : 0.0;
  k_conserved<<<(int)nb, kBlock, 0, s>>>(pos, vel, sp, mt, n, partials, ticket, out_dev);
  return launch_status();
}

}  // extern "C"

// ============================================================= allocation-free LJ force entry point ==
// Some callers cannot allocate device memory when they need forces: code that owns every byte of the GPU
// through its own pool, real-time loops that forbid allocation after start-up, or plug-in hosts that hand
// out only input and output buffers. acs_lj_fp64_noalloc serves them: it runs the same FP64 LJ kernel as
// acs_lj_fp64, but its reduction scratch (one FP64 partial per 256-atom block plus a completion counter)
// lives in the fixed device array below instead of a caller-provided work buffer.
//
// The array is 64 KiB + 256 B and exists on every GPU that loads this library until the process exits;
// it bounds n at kNoAllocMaxAtoms = 2,097,152 atoms. All calls share it, so calls whose work overlaps on the
// GPU (different streams, or different host threads on one device) race and corrupt each other's energy;
// serialise them. The completion counter is cleared at the start of every call; the partials are fully
// overwritten by each call.
namespace {

constexpr int64_t kNoAllocMaxBlocks = 8192;                   // 8192 partials of 8 bytes = 64 KiB
constexpr int64_t kNoAllocMaxAtoms = kNoAllocMaxBlocks * kBlock;  // 2,097,152
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocMaxBlocks * 8 + 256];

// The address is looked up once per CUDA context (the primary context of each device, or any context a driver-API
// caller makes current): a symbol's address belongs to the context the module was loaded into, so a cache keyed
// by the device alone would hand a non-primary context, or a primary context re-created after cudaDeviceReset,
// an address it cannot use.
struct NoAllocEntry {
  int dev;
  void* ctx;
  void* ptr;
};
constexpr int kNoAllocCache = 64;
std::mutex g_noalloc_mutex;
NoAllocEntry g_noalloc_cache[kNoAllocCache];
int g_noalloc_used = 0;

// cuCtxGetCurrent through the runtime's driver entry point (no link against libcuda); null if unavailable.
using CtxGetCurrentFn = int (*)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return (CtxGetCurrentFn)p;
  }();
  return fn;
}

// Device address of g_noalloc_scratch in the current context, looked up on the first call in that context.
// Before the runtime has made a context current, the symbol lookup itself initialises the device's primary
// context, which is then the current one.
int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return ACS_ERR_NO_DEVICE;
  CtxGetCurrentFn get = ctx_get_current();
  void* ctx = nullptr;
  if (!get || get(&ctx) != 0) return ACS_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  for (int k = 0; ctx && k < g_noalloc_used; ++k) {
    if (g_noalloc_cache[k].dev == dev && g_noalloc_cache[k].ctx == ctx) {
      *out = g_noalloc_cache[k].ptr;
      return ACS_OK;
    }
  }
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return ACS_ERR_CUDA;
  if (!ctx && (get(&ctx) != 0 || !ctx)) return ACS_ERR_CUDA;
  if (g_noalloc_used < kNoAllocCache) g_noalloc_cache[g_noalloc_used++] = NoAllocEntry{dev, ctx, p};
  *out = p;
  return ACS_OK;
}

}  // namespace

extern "C" int acs_lj_fp64_noalloc(const double* pos, const int32_t* sp, int64_t n, const double* box3, int periodic,
                                   const int32_t* nbr, const int32_t* nnb, int32_t maxnb, int32_t n_species,
                                   const double* eps_tab, const double* sig_tab, double cutoff, double* force,
                                   double* energy_dev, void* stream) {
  if (n > kNoAllocMaxAtoms) return ACS_ERR_UNSUPPORTED;
  if (n < 1 || !pos || !sp || !force || !energy_dev || !eps_tab || !sig_tab || n_species < 1 ||
      n_species > ACS_MAX_SPECIES || !(cutoff > 0.0) || (nbr && (!nnb || maxnb < 1)))
    return ACS_ERR_ARG;
  void* scratch = nullptr;
  int st = noalloc_scratch(&scratch);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nb = ceil_div(n, kBlock);
  double* partials = (double*)scratch;
  unsigned int* ticket = (unsigned int*)((char*)scratch + kNoAllocMaxBlocks * 8);
  if (cudaMemsetAsync(ticket, 0, 4, s) != cudaSuccess) return ACS_ERR_CUDA;
  LJTab t;
  t.ns = n_species;
  for (int a = 0; a < n_species * n_species; ++a) {
    t.eps[a] = eps_tab[a];
    t.sig2[a] = sig_tab[a] * sig_tab[a];
    const double rc = cutoff * sig_tab[a];
    t.rc2[a] = rc * rc;
  }
  const double c2 = cutoff * cutoff;
  const double src6 = (1.0 / c2) * (1.0 / c2) * (1.0 / c2);
  t.shift6 = src6 * src6 - src6;
  Box3 b = make_box(box3, periodic);
  if (nbr)
    k_lj64<false><<<(int)nb, kBlock, 0, s>>>(pos, sp, n, b, nbr, nnb, maxnb, t, force, partials, ticket, energy_dev);
  else
    k_lj64<true><<<(int)nb, kBlock, 0, s>>>(pos, sp, n, b, nullptr, nullptr, 0, t, force, partials, ticket,
                                           energy_dev);
  return launch_status();
}
