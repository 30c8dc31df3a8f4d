// Device-resident MD engine: FP32-compensated pair forces with FP64 integration, for one system or a
// batch of independent replicas advanced together, captured in CUDA graphs.
//
// Per step the graph runs two kernels:
//   k_step    1 to 32 threads per atom slot: Kahan-compensated FP32 LJ / DSF pair sum over the atom's full
//             neighbour list (DSF exclusions flagged in the entries) -> FP64 acceleration -> second half-kick (step completed; records taken
//             here) -> first half-kick of the next step -> drift -> FP32 image for the next step ->
//             displacement test that flags its replica for a list rebuild. (accusim/integrators.py:25-31
//             with the two kicks of consecutive steps fused.)
//   k_rebuild cooperative, bounded grid barriers; returns at once unless a replica is flagged (or
//             records are due): re-bins flagged replicas into cells of size >= list radius, reorders
//             their atoms by cell, rebuilds the lists with the reference's FP64 pair filter
//             (accusim/forces.py:279-321, :86-98), and reduces per-replica records.
//
// Positions are held as FP64 offsets u from the origin of the cell the atom was binned into at the last
// rebuild (continuous between rebuilds); the absolute wrapped position is py_mod(origin + u, box), as
// accusim/system.py:124-129 keeps it. Pair displacements are d = (img_j - img_i) + m * cell, with the FP32
// images img = float(u) and the integer image shift m in {-1,0,1}^3 stored with the neighbour index
// (entry = slot | code << 27, code = (m0 + 1) + 3 (m1 + 1) + 9 (m2 + 1); with DSF exclusions bit 26 flags an
// excluded pair and the slot takes 26 bits). d_ji == -d_ij bitwise, so pair forces are exactly antisymmetric.
#include <cooperative_groups.h>
#include <math.h>

#include <algorithm>
#include <map>
#include <vector>

#include "accusim_b200_engine.h"
#include "accusim_b200_mlp.h"
#include <cuda_bf16.h>
#include "common.cuh"

using namespace acs;

namespace {

constexpr int kMaxRep = 8192;   // replicas per engine (flag bitmap in shared memory)
constexpr int kRecW = 8;        // KE, PE, Px, Py, Pz, Lx, Ly, Lz
constexpr int kChunkTiles = 64; // record-reduction chunk, in atom groups (G atoms each)
constexpr int kCellChunk = 1024;  // cell-scan chunk (4 cells per thread of a 256-thread block)
constexpr int kIdxBits = 27;
constexpr uint32_t kIdxMask = (1u << kIdxBits) - 1u;
constexpr uint32_t kExBit = 1u << 26;   // with DSF exclusions: flag of an excluded pair in a list entry
constexpr long long kSpinLimit = 20000000;  // default barrier wait: ~2 s of 100 ns sleeps
constexpr int kSmallUnit = 4;   // atoms a warp takes at a time in the list build of one-cell-axis replicas

struct RepDev {
  int64_t atom0;
  int32_t n, npad;
  int32_t cellbase, ncells;  // cell arrays: [cellbase, cellbase + ncells] (last entry is the sentinel)
  int32_t nc[3];
  int32_t tile0, ntiles;
  int32_t chunk0, nchunks;   // record-reduction chunks over this replica's atom groups
  int32_t cc0, ncc;          // cell-scan chunks (kCellChunk cells each)
  double L[3], cs[3];
  float csf[3];
  float pad0;
  double dt, hdt, hs2, rl2;
  double lv_c1, lv_pad;                 // Langevin: exp(-gamma dt)
  double nh_Q, nh_nfkT;                 // Nose-Hoover: thermostat mass, N_f kT
  double lv_sig[ACS_MAX_SPECIES];       // Langevin: sqrt((1 - c1^2) kT / m) per species
};

struct FFDev {
  int ns, lj, dsf, pad;
  float lj_eps4[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float lj_eps24[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float lj_sig2[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  // the same LJ pair in powers of 1/r^2 (the species-pair kernels): F/r = ir2 ir6 (B - A ir6) and
  // U = ir6 (C ir6 - D) - ushift, with A = 48 eps sig^12, B = 24 eps sig^6, C = 4 eps sig^12, D = 4 eps sig^6
  float lj_a[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float lj_b[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float lj_c[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float lj_d[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float lj_rc2[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float lj_ushift[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float qqk[ACS_MAX_SPECIES * ACS_MAX_SPECIES];
  float dsf_a, dsf_rc, dsf_rc2, dsf_c, dsf_erc_rc, dsf_fshift;
  double self_e[ACS_MAX_SPECIES];   // k q^2 (erc/(2 rc) + a/sqrt(pi)) per species
  double mass[ACS_MAX_SPECIES], inv_mass[ACS_MAX_SPECIES];
};

struct Eng {
  int32_t R, maxnb;
  int64_t S;  // slots
  int32_t T, C, nchunks_total;
  int32_t tpa, G, NG;  // threads per atom, atoms per warp (32/tpa), atom groups (S/G)
  RepDev* rep;
  int32_t* active;
  int32_t* flag;
  double *u, *v, *u0, *acc;
  float4* img[2];
  int32_t *cellid, *id, *sp;
  int32_t *nbr, *nnb;
  int32_t *tile_rep, *cell_rep;
  int32_t *chunk_rep, *chunk_tile0, *chunk_ntiles;
  int32_t ncc;
  int32_t *cc_rep, *cc_c0, *cc_n, *cc_sum;
  double *xa, *tmp_xa, *tmp_v;
  int32_t *tmp_cell, *tmp_id, *tmp_sp, *newcell, *perm, *perm2;
  int32_t *count, *start, *cursor;
  // slot order of cells: cells' atoms occupy consecutive slots in the order given by crank (cell id -> position,
  // both global over replicas); start[] is indexed by position, so the atoms of cell c are the slots
  // [start[crank[c]], start[crank[c] + 1]). cell_at is the inverse (position -> cell id).
  int32_t *crank, *cell_at;
  double *partials, *chunk_part, *rec;
  int32_t rec_cap;
  acs_dev_status* status;
  unsigned int* bar;  // [0] counter, [1] generation
  unsigned long long* phase_ns;  // rebuild phase durations, accumulated (block 0 timestamps)
  const float* fext;             // optional per-slot force added to the pair forces (learned correction)
  int32_t thermo;                // 0 VelocityVerlet, 1 Langevin BAOAB, 2 Nose-Hoover
  double* nh_part;               // Nose-Hoover: per atom group sum m v^2
  double* nh_chunk;              // Nose-Hoover: per record chunk sum
  double* nh_st;                 // Nose-Hoover per replica: xi, eta, K2 for the next start half, scale to
                                 // apply, end-half scale (records), 3 spare (8 doubles)
  double* rec_bath;              // bath energy per record and replica
  int32_t* fcell;                // per rebuild: prefix over replicas of the flagged cells the warp-per-cell
                                 // list build covers (R + 1 entries), then that build's cell counter
  int32_t* fsmall;               // the same for the atoms of flagged one-cell-axis replicas, then a unit counter
  int32_t* ftile;                // per rebuild: the flagged replicas' 32-slot tiles (any order), then their count
  const int32_t* ex_start;       // DSF exclusions by atom index within a replica (CSR), or none
  const int32_t* ex_ids;
  int32_t n_ex_ids;
  uint32_t ex_bit;               // list-entry flag of an excluded pair (bit 26), 0 without exclusions
  uint32_t jmask;                // slot bits of a list entry: 26 with exclusions, else 27
  uint32_t seed_lo, seed_hi;
  unsigned long long* octr;      // O-steps taken so far (Langevin draws: counter)
  long long spin_limit;          // polls of a grid-barrier wait before it gives up (0: give up at once)
};

// ------------------------------------------------------------------- Langevin normal draws --
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011): ten rounds of two 32x32->64-bit products with the
// published multipliers, the key bumped by the Weyl constants between rounds.
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
  }
}

// Three standard normals (Box-Muller on u = (x + 1/2) 2^-32) for one atom and one O-step.
__device__ __forceinline__ void langevin_normals(const Eng& E, unsigned long long ostep, int32_t id, int32_t rep,
                                                 double z[3]) {
  uint32_t c[4] = {(uint32_t)ostep, (uint32_t)(ostep >> 32), (uint32_t)id, (uint32_t)rep};
  philox4x32_10(c, E.seed_lo, E.seed_hi);
  const double s32 = 2.3283064365386963e-10;  // 2^-32
  const double u0 = ((double)c[0] + 0.5) * s32, u1 = ((double)c[1] + 0.5) * s32;
  const double u2 = ((double)c[2] + 0.5) * s32, u3 = ((double)c[3] + 0.5) * s32;
  const double r0 = sqrt(-2.0 * log(u0)), r1 = sqrt(-2.0 * log(u2));
  double s0, c0, s1, c1;
  sincospi(2.0 * u1, &s0, &c0);
  sincospi(2.0 * u3, &s1, &c1);
  z[0] = r0 * c0;
  z[1] = r0 * s0;
  z[2] = r1 * c1;
}

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ double py_mod(double x, double L) {
  double r = fmod(x, L);
  if (r != 0.0) {
    if ((L < 0.0) != (r < 0.0)) r = add(r, L);
  } else {
    r = copysign(0.0, L);
  }
  return r;
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
  const float y = x - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// Kahan step for a product term a*b: the product enters the compensated sum through one FMA
// (y = a*b - c rounded once), so the pair force is never rounded on its own.
__device__ __forceinline__ void kahan_fma(float& s, float& c, float a, float b) {
  const float y = fmaf(a, b, -c);
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// Neighbour-list load for the pair loop: read once per step, so it is not kept in L1, which stays with the
// position gathers (measured: the 1M-atom LJ step kernel 0.9% faster than with cache-streaming loads).
__device__ __forceinline__ int32_t ld_list(const int32_t* p) {
  int32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// 1/x by the hardware approximation (relative error within 2^-22), one instruction.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float4 make_img(double ux, double uy, double uz, int sp) {
  return make_float4((float)ux, (float)uy, (float)uz, __int_as_float(sp));
}

__device__ __forceinline__ void cell_coords(int local, const RepDev& R, int& c0, int& c1, int& c2) {
  c2 = local % R.nc[2];
  c1 = (local / R.nc[2]) % R.nc[1];
  c0 = local / (R.nc[2] * R.nc[1]);
}

// ------------------------------------------------------------------------ bounded grid barrier --
// A block that is not the last to arrive polls the generation word up to `limit` times (100 ns apart); if the
// barrier has not opened by then it sets ACS_FLAG_TIMEOUT and returns false, and the caller's kernel returns.
__device__ bool grid_sync(unsigned int* bar, acs_dev_status* st, long long limit) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = bar + 1;
    const unsigned int gen = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(bar, 1u) + 1u;
    ok = 1;
    if (arrived == gridDim.x) {
      bar[0] = 0u;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long it = 0;
      volatile int32_t* vflags = &st->flags;
      while (*vgen == gen) {
        // give up after `limit` polls, or as soon as another block has given up at an earlier barrier
        if (it++ >= limit || ((it & 255) == 0 && (*vflags & ACS_FLAG_TIMEOUT))) {
          atomicOr(&st->flags, ACS_FLAG_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// ------------------------------------------------------------------------------- pair kernel --
// erfc(x), x >= 0, from e = exp(-x^2): Abramowitz & Stegun 7.1.26 (Hastings' approximation, |error| <= 1.5e-7
// in exact arithmetic), erfc(x) = t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) e with t = 1 / (1 + p x). Branch-free
// and it reuses the exponential the DSF force needs anyway; FP32 evaluation stays within 7e-7 of erfc.
__device__ __forceinline__ float erfc_as(float x, float e) {
  const float t = rcp_approx(fmaf(0.3275911f, x, 1.0f));
  const float q = fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f),
                       0.254829592f);
  return t * q * e;
}

// Per-pair coefficients: either the single-species constants (ONE) or the species-pair tables.
struct PairK {
  float eps4, eps24, sig2, a, b, c, d, rc2, ushift, qqk;
};

template <bool ONE>
__device__ __forceinline__ PairK pair_consts(const FFDev& ff, int p, const PairK& c1) {
  if (ONE) return c1;
  PairK k{};
  k.a = ff.lj_a[p];
  k.b = ff.lj_b[p];
  k.c = ff.lj_c[p];
  k.d = ff.lj_d[p];
  k.rc2 = ff.lj_rc2[p];
  k.ushift = ff.lj_ushift[p];
  k.qqk = ff.qqk[p];
  return k;
}

// One pair: accumulate f_i += coef * d (Kahan; with KAHAN false a plain FP32 block partial that the caller
// adds to the Kahan sums) and, when recording, the pair energy (Kahan).
template <bool LJ, bool DSF, bool REC, bool ONE, bool KAHAN = true>
__device__ __forceinline__ void pair_term(const FFDev& ff, const PairK& c1, int sio, const float4& pi, uint32_t e,
                                          const float4& pj, const float4* shift_row, float& fx, float& fy, float& fz,
                                          float& cx, float& cy, float& cz, float& eu, float& ce, uint32_t exb) {
  const float4 sh = shift_row[e >> kIdxBits];
  const float dx = (pj.x - pi.x) + sh.x;
  const float dy = (pj.y - pi.y) + sh.y;
  const float dz = (pj.z - pi.z) + sh.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const PairK k = pair_consts<ONE>(ff, ONE ? 0 : sio + __float_as_int(pj.w), c1);
  float coef = 0.f;
  if (LJ) {  // evaluated for every entry and selected: no divergent branch in the pair loop
    const float ir2 = rcp_approx(r2);
    const bool in = r2 < k.rc2;
    if (ONE) {  // one species: (sig^2/r^2)^3 (the 1M-atom fluid's step is 2% faster with it than below)
      const float sr2 = k.sig2 * ir2;
      const float sr6 = sr2 * sr2 * sr2;
      coef = in ? -k.eps24 * ir2 * sr6 * (2.0f * sr6 - 1.0f) : 0.f;
      if (REC && in) kahan_add(eu, ce, k.eps4 * (sr6 * sr6 - sr6) - k.ushift);
    } else {  // species-pair tables: powers of 1/r^2, two multiplies fewer (4096-ion NaCl step 3% faster)
      const float ir6 = ir2 * ir2 * ir2;
      coef = in ? ir2 * ir6 * fmaf(-k.a, ir6, k.b) : 0.f;
      if (REC && in) kahan_add(eu, ce, ir6 * fmaf(k.c, ir6, -k.d) - k.ushift);
    }
  }
  if (DSF) {  // evaluated for every entry and selected, as the LJ term; excluded pairs (flag exb) have none
    const bool ind = r2 < ff.dsf_rc2 && !(e & exb);
    const float ir = rsqrtf(r2);
    const float rr = r2 * ir;
    const float ar = ff.dsf_a * rr;
    const float ex = __expf(-ar * ar);
    const float er = erfc_as(ar, ex);
    // (erfc(ar)/r^2 + c exp(-(ar)^2)/r - fshift)/r, nested as ((erfc/r + c exp) / r - fshift) / r
    const float cd = k.qqk * (fmaf(fmaf(er, ir, ff.dsf_c * ex), ir, -ff.dsf_fshift) * ir);
    coef -= ind ? cd : 0.f;
    if (REC && ind) kahan_add(eu, ce, k.qqk * (er * ir - ff.dsf_erc_rc + ff.dsf_fshift * (rr - ff.dsf_rc)));
  }
  if (KAHAN) {
    kahan_fma(fx, cx, coef, dx);
    kahan_fma(fy, cy, coef, dy);
    kahan_fma(fz, cz, coef, dz);
  } else {
    fx = fmaf(coef, dx, fx);
    fy = fmaf(coef, dy, fy);
    fz = fmaf(coef, dz, fz);
  }
}

// MODE 0: step (force, kick, record?, kick, drift, image, skin test); 1: last step of a block (force,
// kick, record?, store acceleration); 2: force only (acceleration + records, no kicks).
// A warp handles G = 32/tpa atoms; the tpa lanes of an atom split its neighbour list (lane = phase*G +
// atom-in-group, so each batch of list reads is one coalesced 128-byte row) and their Kahan partial sums
// are combined in FP64 by a fixed xor-shuffle tree (deterministic).
// Second half of a step's start after the first kick: drift (VelocityVerlet), or half drift, the
// Ornstein-Uhlenbeck velocity update and half drift (BAOAB) with the draws of O-step *octr + ostep.
template <bool LV>
__device__ __forceinline__ void drift_or_baoab(const Eng& E, const RepDev& R, int64_t i, int r, int si,
                                               unsigned ostep, double& vx, double& vy, double& vz, double& ux,
                                               double& uy, double& uz) {
  if (LV) {
    ux = E.u[3 * i] + R.hdt * vx;
    uy = E.u[3 * i + 1] + R.hdt * vy;
    uz = E.u[3 * i + 2] + R.hdt * vz;
    double z[3];
    langevin_normals(E, *E.octr + ostep, E.id[i], r, z);
    const double sg = R.lv_sig[si];
    vx = R.lv_c1 * vx + sg * z[0];
    vy = R.lv_c1 * vy + sg * z[1];
    vz = R.lv_c1 * vz + sg * z[2];
    ux += R.hdt * vx;
    uy += R.hdt * vy;
    uz += R.hdt * vz;
  } else {
    ux = E.u[3 * i] + R.dt * vx;
    uy = E.u[3 * i + 1] + R.dt * vy;
    uz = E.u[3 * i + 2] + R.dt * vz;
  }
}

// TH: 0 VelocityVerlet, 1 Langevin BAOAB (the drift of MODE 0 becomes A-O-A), 2 Nose-Hoover (MODE 0 stops
// after the second kick like MODE 1: the thermostat's global kinetic-energy sum comes first; every mode
// writes the group's sum of m v^2 to nh_part).
// PIPE: gathers one block of four entries ahead and list loads two ahead, for step grids under one wave (small
// systems), where occupancy is set by the grid and the extra registers cost nothing; the pair terms are summed
// in the same order, so the results are the same bit for bit.
template <bool LJ, bool DSF, bool REC, int MODE, bool ONE, int TH = 0, bool PIPE = false>
__global__ void __launch_bounds__(256, PIPE ? 1 : 4) k_step(Eng E, FFDev ff, int src, int dst, unsigned ostep) {
  __shared__ float4 shift_tab[8][27];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  if (E.status->flags & (ACS_FLAG_OVERFLOW | ACS_FLAG_NONFINITE | ACS_FLAG_TIMEOUT)) return;
  const float4* __restrict__ imgs = E.img[src];
  // slot bits of a list entry and the DSF exclusion flag (entries of the LJ-only kernel carry no flag)
  const uint32_t jm = DSF ? E.jmask : kIdxMask, exb = DSF ? E.ex_bit : 0u;
  const int G = E.G, tpa = E.tpa;
  const int sub_i = lane % G, phase = lane / G;
  PairK c1{};   // single-species constants (the species-pair kernels read the tables instead)
  c1.eps4 = ff.lj_eps4[0];
  c1.eps24 = ff.lj_eps24[0];
  c1.sig2 = ff.lj_sig2[0];
  c1.rc2 = ff.lj_rc2[0];
  c1.ushift = ff.lj_ushift[0];
  c1.qqk = ff.qqk[0];
  int cur_rep = -1;
  for (int w = blockIdx.x * wpb + wib; w < E.NG; w += gridDim.x * wpb) {
    const int64_t i = (int64_t)w * G + sub_i;
    const int r = E.tile_rep[i >> 5];
    if (!E.active[r]) continue;
    const RepDev& R = E.rep[r];
    if (r != cur_rep) {
      __syncwarp();
      if (lane < 27) {
        const int mx = lane % 3 - 1, my = (lane / 3) % 3 - 1, mz = lane / 9 - 1;
        shift_tab[wib][lane] = make_float4(mx * R.csf[0], my * R.csf[1], mz * R.csf[2], 0.f);
      }
      __syncwarp();
      cur_rep = r;
    }
    const bool valid = (i - R.atom0) < R.n;
    double rv[kRecW] = {0, 0, 0, 0, 0, 0, 0, 0};
    double k2 = 0.0;
    double dfx = 0.0, dfy = 0.0, dfz = 0.0, deu = 0.0;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    int si = 0;
    if (valid) {
      pi = imgs[i];
      si = __float_as_int(pi.w);
      const int sio = si * ACS_MAX_SPECIES;
      const float4* shift_row = shift_tab[wib];
      float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f, eu = 0.f, ce = 0.f;
      const int m = E.nnb[i];
      const int n_it = m > phase ? (m - phase + tpa - 1) / tpa : 0;  // this lane's share of the list
      const int32_t* __restrict__ lst = E.nbr + (int64_t)w * E.maxnb * G + lane;  // entry phase + t*tpa at t*32
      const int n4 = n_it & ~3;
      uint32_t en[4] = {0u, 0u, 0u, 0u}, en2[4] = {0u, 0u, 0u, 0u};
      float4 pjn[4];
      if (n4 > 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) en[q] = (uint32_t)ld_list(lst + q * 32);
        if (PIPE) {
          if (n4 > 4) {
#pragma unroll
            for (int q = 0; q < 4; ++q) en2[q] = (uint32_t)ld_list(lst + (4 + q) * 32);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) pjn[q] = __ldg(imgs + (en[q] & jm));
        }
      }
      int t = 0;
      for (; t < n4; t += 4) {
        uint32_t e[4];
        float4 pj[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) e[q] = en[q];
        if (PIPE) {
          // this block's gathers were issued one block ago; issue the next block's (its entries arrived one
          // block ago) and the list entries of the block after it
#pragma unroll
          for (int q = 0; q < 4; ++q) pj[q] = pjn[q];
#pragma unroll
          for (int q = 0; q < 4; ++q) en[q] = en2[q];
          if (t + 4 < n4) {
#pragma unroll
            for (int q = 0; q < 4; ++q) pjn[q] = __ldg(imgs + (en[q] & jm));
          }
          if (t + 8 < n4) {
#pragma unroll
            for (int q = 0; q < 4; ++q) en2[q] = (uint32_t)ld_list(lst + (t + 8 + q) * 32);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) pj[q] = __ldg(imgs + (e[q] & jm));
          if (t + 4 < n4) {
#pragma unroll
            for (int q = 0; q < 4; ++q) en[q] = (uint32_t)ld_list(lst + (t + 4 + q) * 32);
          }
        }
        // the four pair forces are summed in FP32, the block sum enters the Kahan sums
        float bx = 0.f, by = 0.f, bz = 0.f, bcx, bcy, bcz;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          pair_term<LJ, DSF, REC, ONE, false>(ff, c1, sio, pi, e[q], pj[q], shift_row, bx, by, bz, bcx, bcy, bcz, eu, ce,
                                              exb);
        kahan_add(fx, cx, bx);
        kahan_add(fy, cy, by);
        kahan_add(fz, cz, bz);
      }
      if (t < n_it) {
        // the last 1-3 entries as one more block, their loads issued together; the missing entries get no
        // shift and a partner at 3e30, so r^2 overflows and both terms select zero
        const int rem = n_it - t;
        uint32_t e[4];
        float4 pj[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) e[q] = q < rem ? (uint32_t)ld_list(lst + (t + q) * 32) : (13u << kIdxBits);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          pj[q] = q < rem ? __ldg(imgs + (e[q] & jm)) : make_float4(3e30f, 3e30f, 3e30f, pi.w);
        float bx = 0.f, by = 0.f, bz = 0.f, bcx, bcy, bcz;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          pair_term<LJ, DSF, REC, ONE, false>(ff, c1, sio, pi, e[q], pj[q], shift_row, bx, by, bz, bcx, bcy, bcz, eu, ce,
                                              exb);
        kahan_add(fx, cx, bx);
        kahan_add(fy, cy, by);
        kahan_add(fz, cz, bz);
      }
      dfx = (double)fx - (double)cx;
      dfy = (double)fy - (double)cy;
      dfz = (double)fz - (double)cz;
      deu = (double)eu - (double)ce;
    }
    for (int off = G; off < 32; off <<= 1) {
      dfx += __shfl_xor_sync(0xffffffffu, dfx, off);
      dfy += __shfl_xor_sync(0xffffffffu, dfy, off);
      dfz += __shfl_xor_sync(0xffffffffu, dfz, off);
      if (REC) deu += __shfl_xor_sync(0xffffffffu, deu, off);
    }
    if (valid && phase == 0) {
      if (E.fext) {
        dfx += (double)E.fext[3 * i];
        dfy += (double)E.fext[3 * i + 1];
        dfz += (double)E.fext[3 * i + 2];
      }
      const double im = ff.inv_mass[si];
      const double ax = dfx * im, ay = dfy * im, az = dfz * im;
      if (!(isfinite(ax) && isfinite(ay) && isfinite(az))) atomicOr(&E.status->flags, ACS_FLAG_NONFINITE);
      double vx = E.v[3 * i], vy = E.v[3 * i + 1], vz = E.v[3 * i + 2];
      if (MODE != 2) {
        vx += R.hdt * ax;
        vy += R.hdt * ay;
        vz += R.hdt * az;
      }
      if (REC) {
        const double ms = ff.mass[si];
        rv[0] = 0.5 * ms * (vx * vx + vy * vy + vz * vz);
        rv[1] = 0.5 * deu - (DSF ? ff.self_e[si] : 0.0);
        const double px = ms * vx, py = ms * vy, pz = ms * vz;
        rv[2] = px;
        rv[3] = py;
        rv[4] = pz;
        int c0, c1i, c2;
        cell_coords(E.cellid[i] - R.cellbase, R, c0, c1i, c2);
        const double x = py_mod(c0 * R.cs[0] + E.u[3 * i], R.L[0]);
        const double y = py_mod(c1i * R.cs[1] + E.u[3 * i + 1], R.L[1]);
        const double z = py_mod(c2 * R.cs[2] + E.u[3 * i + 2], R.L[2]);
        rv[5] = y * pz - z * py;
        rv[6] = z * px - x * pz;
        rv[7] = x * py - y * px;
      }
      if (TH == 2) k2 = ff.mass[si] * (vx * vx + vy * vy + vz * vz);
      if (MODE == 0 && TH != 2) {
        vx += R.hdt * ax;
        vy += R.hdt * ay;
        vz += R.hdt * az;
        double ux, uy, uz;
        drift_or_baoab<TH == 1>(E, R, i, r, si, ostep, vx, vy, vz, ux, uy, uz);
        E.u[3 * i] = ux;
        E.u[3 * i + 1] = uy;
        E.u[3 * i + 2] = uz;
        E.img[dst][i] = make_img(ux, uy, uz, si);
        const double ddx = ux - E.u0[3 * i], ddy = uy - E.u0[3 * i + 1], ddz = uz - E.u0[3 * i + 2];
        if (!(ddx * ddx + ddy * ddy + ddz * ddz < R.hs2)) E.flag[r] = 1;
      } else {
        E.acc[3 * i] = ax;
        E.acc[3 * i + 1] = ay;
        E.acc[3 * i + 2] = az;
      }
      if (MODE != 2) {
        E.v[3 * i] = vx;
        E.v[3 * i + 1] = vy;
        E.v[3 * i + 2] = vz;
      }
    }
    if (REC) {
#pragma unroll
      for (int q = 0; q < kRecW; ++q) {
        double x = rv[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) E.partials[(int64_t)w * kRecW + q] = x;
      }
    }
    if (TH == 2) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) k2 += __shfl_down_sync(0xffffffffu, k2, o);
      if (lane == 0) E.nh_part[w] = k2;
    }
  }
}

// ------------------------------------------------------------------------------- Nose-Hoover --
// Per record chunk: the groups' sums of m v^2 in group order (deterministic).
__global__ void k_nh_chunks(Eng E) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < E.nchunks_total; c += gridDim.x * blockDim.x) {
    if (!E.active[E.chunk_rep[c]]) continue;
    double s = 0.0;
    const int t0 = E.chunk_tile0[c], nt = E.chunk_ntiles[c];
    for (int t = 0; t < nt; ++t) s += E.nh_part[t0 + t];
    E.nh_chunk[c] = s;
  }
}

// Thermostat scalars, one thread per replica, with the half-step of accusim/integrators.py:94-103:
//   xi += dt/4 (K2 - N_f kT) / Q;  s = exp(-dt/2 xi);  eta += dt/2 xi;  xi += dt/4 (K2 s^2 - N_f kT) / Q
// (K2 = sum m v^2, the velocities then scale by s). mode 0: initial state (K2 kept for the first start
// half); 1: start half of a block's first step; 2: end half of a block's last step; 3: end half of step k
// then start half of step k + 1 (K2 s1^2 is the scaled velocities' sum). Writes the scale to apply, the
// end-half scale for the records and, on record steps, the bath energy Q xi^2 / 2 + N_f kT eta.
__global__ void k_nh_scalars(Eng E, int mode, int rec, int rec_idx) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= E.R || !E.active[r]) return;
  const RepDev& R = E.rep[r];
  double* st = E.nh_st + 8 * (int64_t)r;
  double xi = st[0], eta = st[1];
  const double dt = R.dt, Q = R.nh_Q, nfkT = R.nh_nfkT;
  auto half = [&](double k2) {
    xi += 0.25 * dt * (k2 - nfkT) / Q;
    const double sc = exp(-0.5 * dt * xi);
    eta += 0.5 * dt * xi;
    xi += 0.25 * dt * (k2 * (sc * sc) - nfkT) / Q;
    return sc;
  };
  double k2 = 0.0;
  if (mode != 1) {
    for (int c = 0; c < R.nchunks; ++c) k2 += E.nh_chunk[R.chunk0 + c];
  }
  // records hold the state after the step's end half (accusim/simulation.py:88 records after the step)
  auto record = [&]() {
    if (rec && rec_idx < E.rec_cap) E.rec_bath[(int64_t)rec_idx * E.R + r] = 0.5 * Q * (xi * xi) + nfkT * eta;
  };
  if (mode == 0) {
    st[2] = k2;
    st[3] = 1.0;
    st[4] = 1.0;
    record();
  } else if (mode == 1) {
    st[3] = half(st[2]);
  } else {
    const double s1 = half(k2);
    const double k2e = k2 * (s1 * s1);
    st[4] = s1;
    record();
    if (mode == 3) {
      st[3] = s1 * half(k2e);
    } else {
      st[3] = s1;
      st[2] = k2e;
    }
  }
  st[0] = xi;
  st[1] = eta;
}

// Sum of m v^2 per atom group (groups of G slots, the step kernel's grouping) from the stored velocities.
__global__ void k_nh_ke(Eng E, FFDev ff) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < E.NG; w += gridDim.x * blockDim.x) {
    double k2 = 0.0;
    for (int q = 0; q < E.G; ++q) {
      const int64_t i = (int64_t)w * E.G + q;
      const int r = E.tile_rep[i >> 5];
      if (!E.active[r] || i - E.rep[r].atom0 >= E.rep[r].n) continue;
      const double vx = E.v[3 * i], vy = E.v[3 * i + 1], vz = E.v[3 * i + 2];
      k2 += ff.mass[E.sp[i]] * (vx * vx + vy * vy + vz * vz);
    }
    E.nh_part[w] = k2;
  }
}

// Apply the thermostat scale per atom; `full`: then the first kick, drift, image and skin test of the next
// step (what k_step's MODE 0 does without a thermostat).
__global__ void k_nh_apply(Eng E, int full, int dst) {
  if (E.status->flags & (ACS_FLAG_OVERFLOW | ACS_FLAG_NONFINITE | ACS_FLAG_TIMEOUT)) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E.S; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = E.tile_rep[i >> 5];
    if (!E.active[r]) continue;
    const RepDev& R = E.rep[r];
    if (i - R.atom0 >= R.n) continue;
    const double sc = E.nh_st[8 * (int64_t)r + 3];
    double vx = sc * E.v[3 * i], vy = sc * E.v[3 * i + 1], vz = sc * E.v[3 * i + 2];
    if (full) {
      vx += R.hdt * E.acc[3 * i];
      vy += R.hdt * E.acc[3 * i + 1];
      vz += R.hdt * E.acc[3 * i + 2];
      const double ux = E.u[3 * i] + R.dt * vx, uy = E.u[3 * i + 1] + R.dt * vy, uz = E.u[3 * i + 2] + R.dt * vz;
      E.u[3 * i] = ux;
      E.u[3 * i + 1] = uy;
      E.u[3 * i + 2] = uz;
      E.img[dst][i] = make_img(ux, uy, uz, E.sp[i]);
      const double ddx = ux - E.u0[3 * i], ddy = uy - E.u0[3 * i + 1], ddz = uz - E.u0[3 * i + 2];
      if (!(ddx * ddx + ddy * ddy + ddz * ddz < R.hs2)) E.flag[r] = 1;
    }
    E.v[3 * i] = vx;
    E.v[3 * i + 1] = vy;
    E.v[3 * i + 2] = vz;
  }
}

// End of a block of `steps` steps: the Langevin draws of the next block continue the O-step count.
__global__ void k_octr_advance(unsigned long long* octr, int steps) { *octr += (unsigned long long)steps; }

// Prologue of a block: first half-kick and drift from the stored accelerations, image, skin test.
__global__ void k_prologue(Eng E, int dst) {
  if (E.status->flags & (ACS_FLAG_OVERFLOW | ACS_FLAG_NONFINITE | ACS_FLAG_TIMEOUT)) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E.S; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = E.tile_rep[i >> 5];
    if (!E.active[r]) continue;
    const RepDev& R = E.rep[r];
    if (i - R.atom0 >= R.n) continue;
    const double sc = E.thermo == 2 ? E.nh_st[8 * (int64_t)r + 3] : 1.0;   // Nose-Hoover start half
    double vx = sc * E.v[3 * i] + R.hdt * E.acc[3 * i];
    double vy = sc * E.v[3 * i + 1] + R.hdt * E.acc[3 * i + 1];
    double vz = sc * E.v[3 * i + 2] + R.hdt * E.acc[3 * i + 2];
    double ux, uy, uz;
    if (E.thermo == 1) drift_or_baoab<true>(E, R, i, r, E.sp[i], 0u, vx, vy, vz, ux, uy, uz);
    else drift_or_baoab<false>(E, R, i, r, E.sp[i], 0u, vx, vy, vz, ux, uy, uz);
    E.v[3 * i] = vx;
    E.v[3 * i + 1] = vy;
    E.v[3 * i + 2] = vz;
    E.u[3 * i] = ux;
    E.u[3 * i + 1] = uy;
    E.u[3 * i + 2] = uz;
    E.img[dst][i] = make_img(ux, uy, uz, E.sp[i]);
    const double ddx = ux - E.u0[3 * i], ddy = uy - E.u0[3 * i + 1], ddz = uz - E.u0[3 * i + 2];
    if (!(ddx * ddx + ddy * ddy + ddz * ddz < R.hs2)) E.flag[r] = 1;
  }
}

__device__ __forceinline__ int wrapc(int c, int nc) { return c < 0 ? c + nc : (c >= nc ? c - nc : c); }

__device__ int block_scan_excl(int v, int* total) {
  __shared__ int ws[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    ws[lane] = w;
  }
  __syncthreads();
  const int ex = x - v + (wid ? ws[wid - 1] : 0);
  *total = ws[(blockDim.x >> 5) - 1];
  __syncthreads();
  return ex;
}

// DSF exclusion of the pair of atoms (a, b), indices within their replica: b among a's excluded atoms
// (accusim/forces.py:418-426).
__device__ __forceinline__ bool dsf_excluded(const Eng& E, int32_t a, int32_t b) {
  if ((uint32_t)a >= (uint32_t)E.n_ex_ids) return false;
  for (int32_t q = E.ex_start[a]; q < E.ex_start[a + 1]; ++q)
    if (E.ex_ids[q] == b) return true;
  return false;
}

// Per-atom state of the list build: stencil ranges, FP32 screen and the exact FP64 decision.
struct PairScan {
  const Eng& E;
  const RepDev& R;
  int64_t i;
  int c[3], lo[3], hi[3];
  bool one[3];
  float4 pi;
  float lo_f, hi_f, Lf[3];
  const float4* im;
  int32_t* lst;

  __device__ PairScan(const Eng& e, const RepDev& r, int64_t atom, int dst) : E(e), R(r), i(atom) {
    cell_coords(E.cellid[i] - R.cellbase, R, c[0], c[1], c[2]);
    im = E.img[dst];
    pi = im[i];
    const float rl2f = (float)R.rl2;
    lo_f = rl2f * (1.0f - 1e-4f);
    hi_f = rl2f * (1.0f + 1e-4f);
    for (int d = 0; d < 3; ++d) {
      Lf[d] = (float)R.L[d];
      one[d] = R.nc[d] < 3;
      lo[d] = one[d] ? 0 : -1;
      hi[d] = one[d] ? 0 : 1;
    }
    lst = E.nbr + (i / E.G) * (int64_t)E.maxnb * E.G + (i % E.G);
  }
  __device__ int cell(int a, int b, int d) const {
    const int n0 = wrapc(c[0] + a, R.nc[0]), n1 = wrapc(c[1] + b, R.nc[1]), n2 = wrapc(c[2] + d, R.nc[2]);
    return R.cellbase + (n0 * R.nc[1] + n1) * R.nc[2] + n2;
  }
  // Exact decision for candidate k: the code to store, or -1. Band candidates use the FP64 filter; others
  // are decided by the FP32 screen (with the FP32 wrap for one-cell axes).
  __device__ int test(int k, int a, int b, int d) const {
    const float4 pj = im[k];
    float x = (pj.x - pi.x) + a * R.csf[0], y = (pj.y - pi.y) + b * R.csf[1], z = (pj.z - pi.z) + d * R.csf[2];
    int w[3] = {0, 0, 0};
    if (one[0]) { w[0] = x > 0.5f * Lf[0] ? 1 : (x < -0.5f * Lf[0] ? -1 : 0); x -= w[0] * Lf[0]; }
    if (one[1]) { w[1] = y > 0.5f * Lf[1] ? 1 : (y < -0.5f * Lf[1] ? -1 : 0); y -= w[1] * Lf[1]; }
    if (one[2]) { w[2] = z > 0.5f * Lf[2] ? 1 : (z < -0.5f * Lf[2] ? -1 : 0); z -= w[2] * Lf[2]; }
    const float q = x * x + y * y + z * z;
    if (!(q < hi_f)) return -1;
    if (q <= lo_f) {
      const int mx = one[0] ? -w[0] : a, my = one[1] ? -w[1] : b, mz = one[2] ? -w[2] : d;
      return (mx + 1) + 3 * (my + 1) + 9 * (mz + 1);
    }
    double dx = sub(E.tmp_xa[3 * k], E.tmp_xa[3 * i]);
    double dy = sub(E.tmp_xa[3 * k + 1], E.tmp_xa[3 * i + 1]);
    double dz = sub(E.tmp_xa[3 * k + 2], E.tmp_xa[3 * i + 2]);
    const int kx = dx > 0.5 * R.L[0] ? 1 : (dx < -0.5 * R.L[0] ? -1 : 0);
    const int ky = dy > 0.5 * R.L[1] ? 1 : (dy < -0.5 * R.L[1] ? -1 : 0);
    const int kz = dz > 0.5 * R.L[2] ? 1 : (dz < -0.5 * R.L[2] ? -1 : 0);
    if (kx) dx = sub(dx, kx > 0 ? R.L[0] : -R.L[0]);
    if (ky) dy = sub(dy, ky > 0 ? R.L[1] : -R.L[1]);
    if (kz) dz = sub(dz, kz > 0 ? R.L[2] : -R.L[2]);
    if (!(norm2(dx, dy, dz) < R.rl2)) return -1;
    const int mx = one[0] ? -kx : a, my = one[1] ? -ky : b, mz = one[2] ? -kz : d;
    return (mx + 1) + 3 * (my + 1) + 9 * (mz + 1);
  }
  __device__ void finish(int cnt) const {
    E.nnb[i] = min(cnt, E.maxnb);
    if (cnt > E.maxnb) {
      atomicOr(&E.status->flags, ACS_FLAG_OVERFLOW);
      atomicMax(&E.status->need_nbr, cnt);
    }
  }
};

// Grid-stride walk over the slots of the rebuild's flagged tiles (listed in phase P0 of this launch, read through
// L2; padding slots excluded), calling f(s, r); with one replica, which is flagged whenever a rebuild runs, over
// all its slots. An ensemble rebuild touches a few % of its slots, which this
// visits without scanning the others; the phases that use it do not depend on the order of the slots.
template <class F>
__device__ __forceinline__ void for_flagged_slots(const Eng& E, int64_t gtid, int64_t gstride, F&& f) {
  if (E.R == 1) {   // one replica, rebuilt: every slot
    for (int64_t s = gtid; s < E.S; s += gstride)
      if (s < E.rep[0].n) f(s, 0);
    return;
  }
  const int64_t nslots = (int64_t)__ldcg(E.ftile + (E.S >> 5)) * 32;
  for (int64_t q = gtid; q < nslots; q += gstride) {
    const int t = __ldcg(E.ftile + (q >> 5));
    const int64_t s = (int64_t)t * 32 + (q & 31);
    const int r = __ldg(E.tile_rep + t);
    if (s - E.rep[r].atom0 < E.rep[r].n) f(s, r);
  }
}

// The list of atom i built by one warp: the lanes take 32 candidates at a time, in stencil order and ascending
// slot, and a ballot keeps the accepted ones in that order.
template <bool EX>
__device__ __forceinline__ void list_atom_warp(const Eng& E, const RepDev& R, int64_t i, int dst, int lane) {
  PairScan ps(E, R, i, dst);
  int cnt = 0;
  for (int a = ps.lo[0]; a <= ps.hi[0]; ++a)
    for (int b = ps.lo[1]; b <= ps.hi[1]; ++b)
      for (int d = ps.lo[2]; d <= ps.hi[2]; ++d) {
        const int cc = ps.cell(a, b, d);
        const int k0 = E.start[E.crank[cc]], k1 = E.start[E.crank[cc] + 1];
        for (int base = k0; base < k1; base += 32) {
          const int k = base + lane;
          int code = -1;
          if (k < k1 && k != i) code = ps.test(k, a, b, d);
          const unsigned bal = __ballot_sync(0xffffffffu, code >= 0);
          const int pos = cnt + __popc(bal & ((1u << lane) - 1u));
          if (code >= 0 && pos < E.maxnb) {
            uint32_t v = (uint32_t)k | ((uint32_t)code << kIdxBits);
            if (EX && dsf_excluded(E, E.id[i], E.id[k])) v |= E.ex_bit;
            ps.lst[(int64_t)pos * E.G] = (int32_t)v;
          }
          cnt += __popc(bal);
        }
      }
  if (lane == 0) ps.finish(cnt);
}

// Exact decision for a candidate in the FP32 band around the list radius, on a replica with >= 3 cells per
// axis: the reference's FP64 filter on the absolute positions (minimum image by comparison with box/2).
// Kept out of line so the candidate loop branches around it instead of issuing it predicated.
__device__ __noinline__ bool band_accept(const double* __restrict__ xa, int64_t i, int64_t k, double L0, double L1,
                                         double L2, double rl2) {
  double dx = sub(xa[3 * k], xa[3 * i]);
  double dy = sub(xa[3 * k + 1], xa[3 * i + 1]);
  double dz = sub(xa[3 * k + 2], xa[3 * i + 2]);
  if (dx > 0.5 * L0) dx = sub(dx, L0); else if (dx < -0.5 * L0) dx = sub(dx, -L0);
  if (dy > 0.5 * L1) dy = sub(dy, L1); else if (dy < -0.5 * L1) dy = sub(dy, -L1);
  if (dz > 0.5 * L2) dz = sub(dz, L2); else if (dz < -0.5 * L2) dz = sub(dz, -L2);
  return norm2(dx, dy, dz) < rl2;
}

// Rebuild of flagged replicas and per-replica record reduction. Cooperative launch (all blocks resident);
// every wait is bounded and reports ACS_FLAG_TIMEOUT instead of hanging. EX: the engine has DSF exclusions
// (excluded pairs' list entries get the flag E.ex_bit).
template <bool EX>
__global__ void __launch_bounds__(256, 3) k_rebuild(Eng E, int dst, int rec, int rec_idx, int force_all) {
  __shared__ unsigned char fl[kMaxRep];
  __shared__ int any_s;
  if (threadIdx.x == 0) any_s = 0;
  __syncthreads();
  int local_any = 0;
  for (int r = threadIdx.x; r < E.R; r += blockDim.x) {
    const unsigned char f = (E.active[r] && (force_all || E.flag[r])) ? 1 : 0;
    fl[r] = f;
    local_any |= f;
  }
  if (local_any) atomicOr(&any_s, 1);
  __syncthreads();
  const bool any = any_s != 0;
  const bool err0 = (E.status->flags & (ACS_FLAG_OVERFLOW | ACS_FLAG_NONFINITE | ACS_FLAG_TIMEOUT)) != 0;
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t gstride = (int64_t)gridDim.x * blockDim.x;

  if (rec && !err0) {
    // Q1: chunk partials (fixed chunking => deterministic)
    for (int c = blockIdx.x; c < E.nchunks_total; c += gridDim.x) {
      if (!E.active[E.chunk_rep[c]]) continue;
      if (threadIdx.x < kRecW) {
        double s = 0.0;
        const int t0 = E.chunk_tile0[c], nt = E.chunk_ntiles[c];
        for (int t = 0; t < nt; ++t) s += E.partials[(int64_t)(t0 + t) * kRecW + threadIdx.x];
        E.chunk_part[(int64_t)c * kRecW + threadIdx.x] = s;
      }
    }
    if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
    // Q2: per-replica sum of its chunks in order
    for (int r = blockIdx.x; r < E.R; r += gridDim.x) {
      if (!E.active[r] || threadIdx.x >= kRecW) continue;
      const RepDev& R = E.rep[r];
      double s = 0.0;
      for (int c = 0; c < R.nchunks; ++c) s += E.chunk_part[(int64_t)(R.chunk0 + c) * kRecW + threadIdx.x];
      if (E.thermo == 2) {  // the partials predate the step's end half: KE scales by s^2, P and L by s
        const double s1 = E.nh_st[8 * (int64_t)r + 4];
        s *= threadIdx.x == 0 ? s1 * s1 : (threadIdx.x == 1 ? 1.0 : s1);
      }
      if (rec_idx < E.rec_cap) E.rec[((int64_t)rec_idx * E.R + r) * kRecW + threadIdx.x] = s;
    }
  }
  if (!any || err0) return;
  unsigned long long t_prev = (blockIdx.x == 0 && threadIdx.x == 0) ? gtimer() : 0ull;
  if (blockIdx.x == 0) {
    // exclusive prefix of the cells the warp-per-cell list build visits (flagged replicas with >= 3 cells on
    // every axis), so that its warps take only those cells (balanced when few replicas rebuild)
    // and of the atoms of flagged replicas with a one-cell axis (the list build's warp-per-atom part)
    const int per = (E.R + blockDim.x - 1) / blockDim.x, r0 = threadIdx.x * per;
    int sum = 0, sum_s = 0;
    for (int r = r0; r < min(r0 + per, E.R); ++r) {
      const RepDev& R = E.rep[r];
      const bool cells3 = R.nc[0] >= 3 && R.nc[1] >= 3 && R.nc[2] >= 3;
      if (fl[r]) {
        if (cells3) sum += R.ncells;
        else sum_s += R.n;
      }
    }
    int total, total_s;
    int ex = block_scan_excl(sum, &total);
    int ex_s = block_scan_excl(sum_s, &total_s);
    for (int r = r0; r < min(r0 + per, E.R); ++r) {
      E.fcell[r] = ex;
      E.fsmall[r] = ex_s;
      const RepDev& R = E.rep[r];
      const bool cells3 = R.nc[0] >= 3 && R.nc[1] >= 3 && R.nc[2] >= 3;
      if (fl[r]) {
        if (cells3) ex += R.ncells;
        else ex_s += R.n;
      }
    }
    if (threadIdx.x == 0) {
      E.fcell[E.R] = total;
      E.fcell[E.R + 1] = 0;   // the list build's cell counter
      E.fsmall[E.R] = total_s;
      E.fsmall[E.R + 1] = 0;  // and its atom-unit counter
      E.ftile[E.S >> 5] = 0;  // the flagged-tile count
    }
  }
#define PHASE(k)                                                  \
  if (blockIdx.x == 0 && threadIdx.x == 0) {                      \
    const unsigned long long t_now = gtimer();                    \
    atomicAdd(&E.phase_ns[k], t_now - t_prev);                    \
    t_prev = t_now;                                               \
  }
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(1);

  // P0: clear counters of flagged replicas' cells; list the flagged replicas' tiles (a warp appends its tiles
  // with one atomic), which the slot phases then walk instead of skipping the unflagged replicas' slots
  for (int64_t c = gtid; c < E.C; c += gstride) {
    if (fl[E.cell_rep[c]]) {
      E.count[c] = 0;
      E.cursor[c] = 0;
    }
  }
  if (E.R > 1) {
    const int lane = threadIdx.x & 31;
    const int64_t T = E.S >> 5;
    for (int64_t t0 = gtid - lane; t0 < T; t0 += gstride) {   // gstride is a multiple of 32: warp-uniform
      const int64_t t = t0 + lane;
      const bool f = t < T && fl[__ldg(E.tile_rep + t)];
      const unsigned bal = __ballot_sync(0xffffffffu, f);
      int base = 0;
      if (lane == 0 && bal) base = atomicAdd(E.ftile + T, __popc(bal));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (f) E.ftile[base + __popc(bal & ((1u << lane) - 1u))] = (int32_t)t;
    }
  }
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(2);
  // P1: absolute wrapped positions and new cells
  for_flagged_slots(E, gtid, gstride, [&](int64_t s, int r) {
    const RepDev& R = E.rep[r];
    int c0, c1, c2;
    cell_coords(E.cellid[s] - R.cellbase, R, c0, c1, c2);
    const double o[3] = {c0 * R.cs[0], c1 * R.cs[1], c2 * R.cs[2]};
    int nc3[3];
    double x[3];
    bool fin = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      x[d] = py_mod(o[d] + E.u[3 * s + d], R.L[d]);
      fin &= isfinite(x[d]);
      // cell = clip(int(x / L * nc), 0, nc - 1)  (accusim/forces.py:290-291)
      const double t = mul(div(x[d], R.L[d]), (double)R.nc[d]);
      nc3[d] = !(t >= 1.0) ? 0 : (t >= (double)(R.nc[d] - 1) ? R.nc[d] - 1 : (int)t);
      E.xa[3 * s + d] = x[d];
    }
    if (!fin) {
      atomicOr(&E.status->flags, ACS_FLAG_NONFINITE);
      nc3[0] = nc3[1] = nc3[2] = 0;
    }
    const int c = R.cellbase + (nc3[0] * R.nc[1] + nc3[1]) * R.nc[2] + nc3[2];
    E.newcell[s] = c;
    atomicAdd(&E.count[c], 1);
  });
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(3);
  // P2: exclusive scan of cell counts -> slot starts, in fixed 1024-cell chunks: (a) chunk-local scans,
  // (b) per-replica prefix of chunk totals (also: sentinel, clear flag, count the rebuild), (c) offsets.
  for (int c = blockIdx.x; c < E.ncc; c += gridDim.x) {
    if (!fl[E.cc_rep[c]]) continue;
    const int c0 = E.cc_c0[c], nc = E.cc_n[c];
    int v[4], sum = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = 4 * threadIdx.x + q;
      v[q] = idx < nc ? E.count[E.cell_at[c0 + idx]] : 0;
      sum += v[q];
    }
    int total;
    int ex = block_scan_excl(sum, &total);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = 4 * threadIdx.x + q;
      if (idx < nc) E.start[c0 + idx] = ex;
      ex += v[q];
    }
    if (threadIdx.x == 0) E.cc_sum[c] = total;
  }
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(4);
  // (b) a block per flagged replica scans its chunk totals (exclusive, from the replica's first slot)
  for (int r = blockIdx.x; r < E.R; r += gridDim.x) {
    if (!fl[r]) continue;
    const RepDev& R = E.rep[r];
    int carry = 0;
    for (int c0 = 0; c0 < R.ncc; c0 += blockDim.x) {
      const int c = c0 + (int)threadIdx.x;
      const int t = c < R.ncc ? E.cc_sum[R.cc0 + c] : 0;
      int total;
      const int ex = block_scan_excl(t, &total);
      if (c < R.ncc) E.cc_sum[R.cc0 + c] = (int32_t)(R.atom0 + carry + ex);
      carry += total;
    }
    if (threadIdx.x == 0) {
      E.start[R.cellbase + R.ncells] = (int32_t)(R.atom0 + R.n);
      E.flag[r] = 0;
      atomicAdd(&E.status->rebuilds, 1);
    }
  }
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(5);
  for (int c = blockIdx.x; c < E.ncc; c += gridDim.x) {
    if (!fl[E.cc_rep[c]]) continue;
    const int c0 = E.cc_c0[c], nc = E.cc_n[c], add_v = E.cc_sum[c];
    for (int idx = threadIdx.x; idx < nc; idx += blockDim.x) E.start[c0 + idx] += add_v;
  }
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(6);
  // P3: scatter old slots to new slots
  for_flagged_slots(E, gtid, gstride, [&](int64_t s, int) {
    const int c = E.newcell[s];
    E.perm[E.start[E.crank[c]] + atomicAdd(&E.cursor[c], 1)] = (int32_t)s;
  });
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(7);
  // P3b: deterministic order inside each cell: every atom's rank among its cell's atoms by old slot
  for_flagged_slots(E, gtid, gstride, [&](int64_t k, int) {
    const int v = E.perm[k];
    const int c = E.newcell[v];
    const int a0 = E.start[E.crank[c]], a1 = E.start[E.crank[c] + 1];
    int rank = 0;
    for (int a = a0; a < a1; ++a) rank += (E.perm[a] < v);
    E.perm2[a0 + rank] = v;
  });
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(8);
  // P4: gather into new order
  for_flagged_slots(E, gtid, gstride, [&](int64_t k, int) {
    const int o = E.perm2[k];
    E.tmp_cell[k] = E.newcell[o];
    E.tmp_id[k] = E.id[o];
    E.tmp_sp[k] = E.sp[o];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      E.tmp_xa[3 * k + d] = E.xa[3 * o + d];
      E.tmp_v[3 * k + d] = E.v[3 * o + d];
    }
  });
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(9);
  // P5: commit; offsets from the new cell origins; images
  for_flagged_slots(E, gtid, gstride, [&](int64_t k, int r) {
    const RepDev& R = E.rep[r];
    const int c = E.tmp_cell[k];
    int c0, c1, c2;
    cell_coords(c - R.cellbase, R, c0, c1, c2);
    const double ux = E.tmp_xa[3 * k] - c0 * R.cs[0];
    const double uy = E.tmp_xa[3 * k + 1] - c1 * R.cs[1];
    const double uz = E.tmp_xa[3 * k + 2] - c2 * R.cs[2];
    E.cellid[k] = c;
    E.id[k] = E.tmp_id[k];
    E.sp[k] = E.tmp_sp[k];
    E.u[3 * k] = ux;
    E.u[3 * k + 1] = uy;
    E.u[3 * k + 2] = uz;
    E.u0[3 * k] = ux;
    E.u0[3 * k + 1] = uy;
    E.u0[3 * k + 2] = uz;
#pragma unroll
    for (int d = 0; d < 3; ++d) E.v[3 * k + d] = E.tmp_v[3 * k + d];
    E.img[dst][k] = make_img(ux, uy, uz, E.tmp_sp[k]);
  });
  if (!grid_sync(E.bar, E.status, E.spin_limit)) return;
  PHASE(10);
  // P6: neighbour lists in one pass over the 27-cell stencil. Each candidate's r^2 is first computed in
  // FP32 from the new images (relative error ~1e-6): outside rl^2 (1 + 1e-4) it is rejected, inside
  // rl^2 (1 - 1e-4) accepted; only the band between is decided by the reference's FP64 filter. So the
  // pair set is exactly the FP64 filter's. That filter takes the minimum image by comparison with box/2,
  // which for every pair that can lie inside the list radius (< box/2) is the IEEE result of
  // d - box*round(d/box). The image shift stored with j is the stencil offset (>= 3 cells per edge) or
  // minus the wrap (1 cell per edge). Entries are in stencil order, ascending slot within a cell, however
  // the work is split: a warp per atom when the pair kernel runs >= 8 threads per atom (small systems), else a
  // warp per home cell, and a warp per atom for replicas with a one-cell axis.
  if (E.tpa >= 8) {
    const int64_t gw = gtid >> 5, nw = gstride >> 5;
    const int lane = threadIdx.x & 31;
    for (int64_t i = gw; i < E.S; i += nw) {
      const int r = E.tile_rep[i >> 5];
      if (!fl[r]) continue;
      const RepDev& R = E.rep[r];
      if (i - R.atom0 >= R.n) continue;
      list_atom_warp<EX>(E, R, i, dst, lane);
    }
  } else {
    // Replicas with >= 3 cells on every axis: a warp per home cell (a warp takes the next of the flagged
    // replicas' cells from a counter, through the prefix block 0 wrote at the start). The candidates of the 27 stencil cells, in
    // list order (stencil cell, then ascending slot), are read 32 at a time with the cell pair's image shift
    // already added; those whose distance to the home cell's box exceeds the list radius (with the band
    // margin) cannot pair with any home atom and are dropped, the rest are compacted in order into a
    // shared-memory buffer. Each full batch of 32 is screened against the home atoms (up to 32, staged in
    // shared memory): for home atom h, two ballots over the batch give its masks (accepted / inside the
    // upper band edge), which lane h keeps. The next raw chunk is loaded while a batch is screened; only the
    // FP64 band decision branches.
    // home atoms' negated coordinates, one array per axis: two adjacent home atoms load as one packed FP32 pair
    __shared__ __align__(8) float hnx[8][32], hny[8][32], hnz[8][32];
    __shared__ float4 bufp[8][64];
    __shared__ uint32_t bufk[8][64];
    __shared__ int selfpos[8][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int nflag = __ldcg(E.fcell + E.R);   // written by block 0 in this launch: read through L2
    // each warp takes the next flagged cell from a counter (cleared by block 0 with the prefix), so warps that
    // drew cheap cells take more: cell costs vary several-fold (occupancy, cell edge per replica)
    auto next_cell = [&]() {
      int v = 0;
      if (lane == 0) v = atomicAdd(E.fcell + E.R + 1, 1);
      return __shfl_sync(0xffffffffu, v, 0);
    };
    for (int f = next_cell(); f < nflag; f = next_cell()) {
      int r = 0;   // the replica whose range of the prefix holds f: the last r with fcell[r] <= f
      for (int lo = 0, hi = E.R - 1; lo <= hi;) {
        const int mid = (lo + hi) >> 1;
        if (__ldcg(E.fcell + mid) <= f) {
          r = mid;
          lo = mid + 1;
        } else {
          hi = mid - 1;
        }
      }
      const RepDev& R = E.rep[r];
      const int64_t c = E.cell_at[R.cellbase + (f - __ldcg(E.fcell + r))];   // home cells in slot order
      const float4* __restrict__ im = E.img[dst];
      const float rl2f = (float)R.rl2, lo_f = rl2f * (1.0f - 1e-4f), hi_f = rl2f * (1.0f + 1e-4f);
      // stencil cell st = 9 (a + 1) + 3 (b + 1) + (d + 1) in list order: lane st holds its first slot, its
      // length and the exclusive prefix P of the lengths (its first position in the packed sequence)
      int sk0 = 0, slen = 0;
      if (lane < 27) {
        int c0, c1, c2;
        cell_coords((int)(c - R.cellbase), R, c0, c1, c2);
        const int n0 = wrapc(c0 + lane / 9 - 1, R.nc[0]), n1 = wrapc(c1 + (lane / 3) % 3 - 1, R.nc[1]),
                  n2 = wrapc(c2 + lane % 3 - 1, R.nc[2]);
        const int cc = R.cellbase + (n0 * R.nc[1] + n1) * R.nc[2] + n2;
        sk0 = E.start[E.crank[cc]];
        slen = E.start[E.crank[cc] + 1] - sk0;
      }
      int incl = slen;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      const int P = incl - slen;
      const int T = __shfl_sync(0xffffffffu, incl, 26);
      const int h0 = __shfl_sync(0xffffffffu, sk0, 13), hn = __shfl_sync(0xffffffffu, slen, 13);
      // this lane's raw candidate at packed position pb + lane: shifted position, list entry (slot | code)
      // and whether it can reach the home cell's box [0, cs)^3 within the list radius
      auto stage = [&](int pb, float4& cp, uint32_t& ck, bool& keep) {
        const int p = pb + lane;
        const int pp = p < T ? p : T - 1;
        int st = 0;   // last stencil cell with P <= pp
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int cs = st + step;
          const int Pc = __shfl_sync(0xffffffffu, P, cs < 27 ? cs : 26);
          if (cs < 27 && Pc <= pp) st = cs;
        }
        const int k = __shfl_sync(0xffffffffu, sk0, st) + (pp - __shfl_sync(0xffffffffu, P, st));
        keep = false;
        ck = 0u;
        cp = make_float4(0.f, 0.f, 0.f, 0.f);
        if (p < T) {
          const int a = st / 9 - 1, b = (st / 3) % 3 - 1, d = st % 3 - 1;
          const float4 pj = im[k];
          cp = make_float4(pj.x + a * R.csf[0], pj.y + b * R.csf[1], pj.z + d * R.csf[2], 0.f);
          ck = (uint32_t)k | ((uint32_t)((a + 1) + 3 * (b + 1) + 9 * (d + 1)) << kIdxBits);
          const float gx = fmaxf(fmaxf(-cp.x, cp.x - R.csf[0]), 0.f);
          const float gy = fmaxf(fmaxf(-cp.y, cp.y - R.csf[1]), 0.f);
          const float gz = fmaxf(fmaxf(-cp.z, cp.z - R.csf[2]), 0.f);
          keep = gx * gx + gy * gy + gz * gz < hi_f;
        }
      };
      for (int hb = 0; hb < hn; hb += 32) {
        const int nh = min(32, hn - hb);
        const bool own = lane < nh;
        const int64_t i = h0 + hb + (own ? lane : 0);
        const uint32_t hlo = (uint32_t)(h0 + hb);
        __syncwarp();
        {
          const float4 hp = im[i];
          hnx[wib][lane] = -hp.x;
          hny[wib][lane] = -hp.y;
          hnz[wib][lane] = -hp.z;
        }
        int32_t* __restrict__ lst = E.nbr + (i / E.G) * (int64_t)E.maxnb * E.G + (i % E.G);
        int cnt = 0, nbuf = 0, rb = 0;
        float4 rp;
        uint32_t rk;
        bool rkeep;
        stage(0, rp, rk, rkeep);
        while (true) {
          if (rb < T) {   // append this raw chunk's survivors, in order
            const unsigned bal = __ballot_sync(0xffffffffu, rkeep);
            if (rkeep) {
              const int pos = nbuf + __popc(bal & lt_mask);
              bufp[wib][pos] = rp;
              bufk[wib][pos] = rk;
            }
            nbuf += __popc(bal);
            rb += 32;
            if (rb < T) stage(rb, rp, rk, rkeep);   // in flight while a batch is screened
          }
          if (nbuf == 0 && rb >= T) break;
          if (nbuf < 32 && rb < T) continue;
          const int nk = min(32, nbuf);
          __syncwarp();
          float4 cur = make_float4(3e30f, 3e30f, 3e30f, 0.f);   // padding: r^2 overflows, never accepted
          uint32_t ck = 0u;
          if (lane < nk) {
            cur = bufp[wib][lane];
            ck = bufk[wib][lane];
          }
          selfpos[wib][lane] = -1;
          __syncwarp();
          const uint32_t hs = (ck & kIdxMask) - hlo;   // home index of this candidate, if it is a home atom
          if (lane < nk && hs < (uint32_t)nh) selfpos[wib][hs] = lane;
          uint32_t m_in = 0u, m_hi = 0u;
          // two home atoms per packed FP32 operation (each half is the IEEE scalar operation); with an odd count
          // the last pair's second atom is a staged non-home slot, whose masks are cleared below
          const float2 px = make_float2(cur.x, cur.x), py = make_float2(cur.y, cur.y), pz = make_float2(cur.z, cur.z);
#pragma unroll 2
          for (int h = 0; h < nh; h += 2) {
            const float2 x = __fadd2_rn(px, *reinterpret_cast<const float2*>(&hnx[wib][h]));
            const float2 y = __fadd2_rn(py, *reinterpret_cast<const float2*>(&hny[wib][h]));
            const float2 z = __fadd2_rn(pz, *reinterpret_cast<const float2*>(&hnz[wib][h]));
            const float2 q = __ffma2_rn(z, z, __ffma2_rn(y, y, __fmul2_rn(x, x)));
            const unsigned bi0 = __ballot_sync(0xffffffffu, q.x <= lo_f), bh0 = __ballot_sync(0xffffffffu, q.x < hi_f);
            const unsigned bi1 = __ballot_sync(0xffffffffu, q.y <= lo_f), bh1 = __ballot_sync(0xffffffffu, q.y < hi_f);
            if (lane == h) {
              m_in = bi0;
              m_hi = bh0;
            }
            if (lane == h + 1) {
              m_in = bi1;
              m_hi = bh1;
            }
          }
          __syncwarp();
          const int self = selfpos[wib][lane];   // never the atom itself
          if (self >= 0) {
            m_in &= ~(1u << self);
            m_hi &= ~(1u << self);
          }
          if (!own) m_in = m_hi = 0u;
          uint32_t m_band = m_hi & ~m_in;
          if (__any_sync(0xffffffffu, m_band != 0u)) {
            while (m_band) {
              const int t = __ffs(m_band) - 1;
              m_band &= m_band - 1u;
              if (band_accept(E.tmp_xa, i, bufk[wib][t] & kIdxMask, R.L[0], R.L[1], R.L[2], R.rl2)) m_in |= 1u << t;
            }
          }
          while (m_in) {   // list order
            const int t = __ffs(m_in) - 1;
            m_in &= m_in - 1u;
            if (cnt < E.maxnb) {
              uint32_t v = bufk[wib][t];
              if (EX && dsf_excluded(E, E.id[i], E.id[v & kIdxMask])) v |= E.ex_bit;
              lst[(int64_t)cnt * E.G] = (int32_t)v;
            }
            ++cnt;
          }
          // keep the survivors beyond this batch at the front of the buffer
          __syncwarp();
          const int rest = nbuf - nk;
          float4 mp = make_float4(0.f, 0.f, 0.f, 0.f);
          uint32_t mk = 0u;
          if (lane < rest) {
            mp = bufp[wib][nk + lane];
            mk = bufk[wib][nk + lane];
          }
          __syncwarp();
          if (lane < rest) {
            bufp[wib][lane] = mp;
            bufk[wib][lane] = mk;
          }
          nbuf = rest;
        }
        if (own) {
          E.nnb[i] = min(cnt, E.maxnb);
          if (cnt > E.maxnb) {
            atomicOr(&E.status->flags, ACS_FLAG_OVERFLOW);
            atomicMax(&E.status->need_nbr, cnt);
          }
        }
      }
    }
    // Replicas with a one-cell axis (small boxes, cells of the whole edge): a warp per atom, the per-axis wrap in
    // the pair test. Warps take units of kSmallUnit atoms in turn from a counter, through a prefix of the flagged
    // small replicas' atom counts that block 0 wrote at the start.
    const int nsmall = __ldcg(E.fsmall + E.R);
    auto next_unit = [&]() {
      int v = 0;
      if (lane == 0) v = atomicAdd(E.fsmall + E.R + 1, 1);
      return __shfl_sync(0xffffffffu, v, 0);
    };
    for (int u = next_unit(); u < (nsmall + kSmallUnit - 1) / kSmallUnit; u = next_unit()) {
      const int q0 = u * kSmallUnit, q1 = min(q0 + kSmallUnit, nsmall);
      int r = 0;   // the last r with fsmall[r] <= q0: the replica that holds atom q0 of the prefix
      for (int lo = 0, hi = E.R - 1; lo <= hi;) {
        const int mid = (lo + hi) >> 1;
        if (__ldcg(E.fsmall + mid) <= q0) {
          r = mid;
          lo = mid + 1;
        } else {
          hi = mid - 1;
        }
      }
      for (int q = q0; q < q1; ++q) {
        while (r + 1 < E.R && __ldcg(E.fsmall + r + 1) <= q) ++r;
        const RepDev& R = E.rep[r];
        list_atom_warp<EX>(E, R, R.atom0 + (q - __ldcg(E.fsmall + r)), dst, lane);
      }
    }
  }
  __syncthreads();
  PHASE(15);
#undef PHASE
}

// Scatter caller arrays (replica-concatenated, engine units) into slots; cell 0 origin so u = x.
__global__ void k_load(Eng E, const double* __restrict__ pos, const double* __restrict__ vel,
                       const int32_t* __restrict__ sp, const int64_t* __restrict__ src0) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < E.S; s += (int64_t)gridDim.x * blockDim.x) {
    const int r = E.tile_rep[s >> 5];
    const RepDev& R = E.rep[r];
    const int64_t loc = s - R.atom0;
    if (loc >= R.n) {
      for (int d = 0; d < 3; ++d) E.u[3 * s + d] = E.v[3 * s + d] = E.u0[3 * s + d] = E.acc[3 * s + d] = 0.0;
      E.id[s] = -1;
      E.sp[s] = 0;
      E.cellid[s] = R.cellbase;
      E.nnb[s] = 0;
      E.img[0][s] = E.img[1][s] = make_float4(0.f, 0.f, 0.f, 0.f);
      continue;
    }
    const int64_t g = src0[r] + loc;
    for (int d = 0; d < 3; ++d) {
      E.u[3 * s + d] = pos[3 * g + d];
      E.v[3 * s + d] = vel[3 * g + d];
      E.acc[3 * s + d] = 0.0;
    }
    E.id[s] = (int32_t)loc;
    E.sp[s] = sp[g];
    E.cellid[s] = R.cellbase;
  }
}

// Gather slots back to caller order: absolute wrapped positions, velocities, accelerations.
__global__ void k_store(Eng E, double* __restrict__ pos, double* __restrict__ vel, double* __restrict__ acc,
                        const int64_t* __restrict__ src0) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < E.S; s += (int64_t)gridDim.x * blockDim.x) {
    const int r = E.tile_rep[s >> 5];
    const RepDev& R = E.rep[r];
    if (s - R.atom0 >= R.n) continue;
    const int64_t g = src0[r] + E.id[s];
    int c0, c1, c2;
    cell_coords(E.cellid[s] - R.cellbase, R, c0, c1, c2);
    const double o[3] = {c0 * R.cs[0], c1 * R.cs[1], c2 * R.cs[2]};
    for (int d = 0; d < 3; ++d) {
      if (pos) pos[3 * g + d] = py_mod(o[d] + E.u[3 * s + d], R.L[d]);
      if (vel) vel[3 * g + d] = E.v[3 * s + d];
      if (acc) acc[3 * g + d] = E.acc[3 * s + d];
    }
  }
}

// Load caller-order state into the current slots without re-binning: offsets stay continuous (minimum
// image against the current offset), so the next block's skin test decides whether the list survives.
__global__ void k_load_keep(Eng E, const double* __restrict__ pos, const double* __restrict__ vel,
                            const int64_t* __restrict__ src0) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < E.S; s += (int64_t)gridDim.x * blockDim.x) {
    const int r = E.tile_rep[s >> 5];
    const RepDev& R = E.rep[r];
    if (s - R.atom0 >= R.n) continue;
    const int64_t g = src0[r] + E.id[s];
    int c0, c1, c2;
    cell_coords(E.cellid[s] - R.cellbase, R, c0, c1, c2);
    const double o[3] = {c0 * R.cs[0], c1 * R.cs[1], c2 * R.cs[2]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double uo = E.u[3 * s + d];
      double du = (pos[3 * g + d] - o[d]) - uo;
      du -= R.L[d] * rint(du / R.L[d]);
      E.u[3 * s + d] = uo + du;
      E.v[3 * s + d] = vel[3 * g + d];
    }
  }
}

// Unique pairs inside the physical cutoffs (LJ r < cutoff sigma_ij, DSF r < rc), by the step kernel's
// FP32 test on the current images: the unit of work for the roofline.
__global__ void k_count_pairs(Eng E, FFDev ff, int src, unsigned long long* out) {
  unsigned long long nl = 0, nd = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E.S; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = E.tile_rep[i >> 5];
    const RepDev& R = E.rep[r];
    if (i - R.atom0 >= R.n) continue;
    const float4 pi = E.img[src][i];
    const int sio = __float_as_int(pi.w) * ACS_MAX_SPECIES;
    const int32_t* lst = E.nbr + (i / E.G) * (int64_t)E.maxnb * E.G + (i % E.G);
    for (int k = 0; k < E.nnb[i]; ++k) {
      const uint32_t e = (uint32_t)lst[(int64_t)k * E.G];
      const float4 pj = E.img[src][e & E.jmask];
      const uint32_t code = e >> kIdxBits;
      const int mx = (int)(code % 3) - 1, my = (int)((code / 3) % 3) - 1, mz = (int)(code / 9) - 1;
      const float dx = (pj.x - pi.x) + mx * R.csf[0];
      const float dy = (pj.y - pi.y) + my * R.csf[1];
      const float dz = (pj.z - pi.z) + mz * R.csf[2];
      const float r2 = dx * dx + dy * dy + dz * dz;
      const int p = sio + __float_as_int(pj.w);
      if (ff.lj && r2 < ff.lj_rc2[p]) ++nl;
      if (ff.dsf && r2 < ff.dsf_rc2 && !(e & E.ex_bit)) ++nd;
    }
  }
  atomicAdd(out, nl);
  atomicAdd(out + 1, nd);
}

// Every neighbour-list entry as a directed pair of caller indices, key = 2 (gi n_total + gj) + excluded (the DSF
// exclusion flag of the entry), and the FP64 absolute positions the lists were built from (the last rebuild's
// wrapped positions, which its exact pair filter used), in caller order. Each slot reserves its entries with one
// atomic; keys beyond `cap` are counted but not written. Order is not deterministic: the caller sorts.
__global__ void k_dump_lists(Eng E, const int64_t* __restrict__ src0, int64_t n_total, long long* __restrict__ keys,
                             long long cap, unsigned long long* __restrict__ count, double* __restrict__ pos_build) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E.S; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = E.tile_rep[i >> 5];
    const RepDev& R = E.rep[r];
    if (i - R.atom0 >= R.n) continue;
    const int64_t gi = src0[r] + E.id[i];
    if (pos_build) {
#pragma unroll
      for (int d = 0; d < 3; ++d) pos_build[3 * gi + d] = E.tmp_xa[3 * i + d];
    }
    const int m = E.nnb[i];
    const unsigned long long base = atomicAdd(count, (unsigned long long)m);
    const int32_t* lst = E.nbr + (i / E.G) * (int64_t)E.maxnb * E.G + (i % E.G);
    for (int k = 0; k < m; ++k) {
      const uint32_t e = (uint32_t)lst[(int64_t)k * E.G];
      const int64_t j = (int64_t)(e & E.jmask);
      const bool own = j < E.S && E.tile_rep[j >> 5] == r && j - R.atom0 < R.n;
      const int64_t gj = own ? src0[r] + E.id[j] : -1;   // -1: an entry naming no atom of this replica
      const long long key = gj < 0 ? -1ll : 2ll * (gi * n_total + gj) + ((e & E.ex_bit) ? 1 : 0);
      if (base + k < (unsigned long long)cap) keys[base + k] = key;
    }
  }
}

// Radial descriptors of every slot from the engine's own images and neighbour lists (FP32), in slot order,
// for the learned force correction: warp per slot, lane = Gaussian channel (definitions as in mlp.cu).
struct DescP {
  float r0, dmu, inv2s2, rc2, pi_rc;
};

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__global__ void __launch_bounds__(256, 4) k_desc_engine(Eng E, int src, DescP P, const float* __restrict__ mean,
                                                      const float* __restrict__ inv_std, __nv_bfloat16* __restrict__ X,
                                                      float* __restrict__ V) {
  // Per pass, 4 chunks of 32 neighbours: (1) lanes split the neighbours (list entries, then positions, each
  // batch of loads in flight together) and stage r, the unit vector, fc and species of those inside the
  // descriptor cutoff in shared memory, in list order; (2) each lane (one Gaussian channel) accumulates over
  // the staged neighbours.
  constexpr int kU = 4;
  __shared__ float4 stage[8][32 * kU];   // (dx/r, dy/r, dz/r, r) per neighbour
  __shared__ float stage2[8][32 * kU];   // log2(fc)
  __shared__ float4 shift_tab[8][27];    // image shift of each stencil code, this warp's replica
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= E.S) return;
  const int r = E.tile_rep[i >> 5];
  const RepDev& R = E.rep[r];
  const bool valid = E.active[r] && (i - R.atom0 < R.n);
  float d[2] = {0.f, 0.f}, vx[2] = {0.f, 0.f}, vy[2] = {0.f, 0.f}, vz[2] = {0.f, 0.f};
  int si = 0;
  if (valid) {
    const float4* __restrict__ im = E.img[src];
    const float4 pi = im[i];
    si = __float_as_int(pi.w);
    const float mu = P.r0 + lane * P.dmu;
    const int m = E.nnb[i];
    const int32_t* lst = E.nbr + (i / E.G) * (int64_t)E.maxnb * E.G + (i % E.G);
    if (lane < 27)
      shift_tab[wib][lane] = make_float4((lane % 3 - 1) * R.csf[0], ((lane / 3) % 3 - 1) * R.csf[1],
                                         (lane / 9 - 1) * R.csf[2], 0.f);
    __syncwarp();
    for (int base = 0; base < m; base += 32 * kU) {
      uint32_t e[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int k = base + 32 * u + lane;
        e[u] = k < m ? (uint32_t)lst[(int64_t)k * E.G] : 0u;
      }
      float4 pj[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int k = base + 32 * u + lane;
        pj[u] = k < m ? im[e[u] & E.jmask] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      // species 0 staged from the front, species 1 from the back, each in list order
      int cnt0 = 0, cnt1 = 0;
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int k = base + 32 * u + lane;
        const float4 sh = shift_tab[wib][e[u] >> kIdxBits];
        const float fx = (pj[u].x - pi.x) + sh.x;
        const float fy = (pj[u].y - pi.y) + sh.y;
        const float fz = (pj[u].z - pi.z) + sh.z;
        const float r2 = fx * fx + fy * fy + fz * fz;
        const bool inside = k < m && r2 < P.rc2;
        const bool s1 = (__float_as_int(pj[u].w) & 1) != 0;
        const unsigned b0 = __ballot_sync(0xffffffffu, inside && !s1), b1 = __ballot_sync(0xffffffffu, inside && s1);
        if (inside) {
          const float ir = rsqrtf(r2), rr = r2 * ir;
          const unsigned lt = (1u << lane) - 1u;
          const int pos = s1 ? (32 * kU - 1) - (cnt1 + __popc(b1 & lt)) : cnt0 + __popc(b0 & lt);
          stage[wib][pos] = make_float4(fx * ir, fy * ir, fz * ir, rr);
          // the cosine cutoff enters the exponent: g fc = 2^(-(r - mu)^2 k log2(e) + log2(fc))
          stage2[wib][pos] = __log2f(0.5f * (__cosf(P.pi_rc * rr) + 1.0f));
        }
        cnt0 += __popc(b0);
        cnt1 += __popc(b1);
      }
      __syncwarp();
      const float k2 = P.inv2s2 * 1.4426950408889634f;
#pragma unroll 4
      for (int q = 0; q < cnt0; ++q) {
        const float4 a = stage[wib][q];
        const float t = a.w - mu;
        const float g = ex2_approx(fmaf(-t * t, k2, stage2[wib][q]));
        d[0] += g; vx[0] = fmaf(g, a.x, vx[0]); vy[0] = fmaf(g, a.y, vy[0]); vz[0] = fmaf(g, a.z, vz[0]);
      }
#pragma unroll 4
      for (int q = 32 * kU - cnt1; q < 32 * kU; ++q) {
        const float4 a = stage[wib][q];
        const float t = a.w - mu;
        const float g = ex2_approx(fmaf(-t * t, k2, stage2[wib][q]));
        d[1] += g; vx[1] = fmaf(g, a.x, vx[1]); vy[1] = fmaf(g, a.y, vy[1]); vz[1] = fmaf(g, a.z, vz[1]);
      }
      __syncwarp();
    }
  }
  __nv_bfloat16* xrow = X + i * 80;
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int c = 32 * s + lane;
    xrow[c] = __float2bfloat16(valid ? (d[s] - mean[c]) * inv_std[c] : 0.f);
    float* vrow = V + (i * 64 + c) * 3;
    vrow[0] = vx[s];
    vrow[1] = vy[s];
    vrow[2] = vz[s];
  }
  if (lane < 16) {
    float v = 0.f;
    if (valid && lane < 2) v = (si == lane) ? 1.f : 0.f;
    if (valid && lane == 15) v = 1.f;
    xrow[64 + lane] = __float2bfloat16(v);
  }
}

inline size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

// ====================================================================================== host side ==
struct acs_engine {
  Eng E;
  FFDev ff;
  std::vector<RepDev> reps;
  std::vector<int64_t> src0;
  int64_t* src0_dev = nullptr;
  int coop_blocks = 0;
  int step_blocks = 0;
  int step_threads = 256;
  bool pipe = false;   // plain steps with gathers one block ahead (step grids under one wave)
  int n_lj = 0, n_dsf = 0;
  std::map<long long, cudaGraphExec_t> graphs;
  int dev = 0;
  // learned force correction (optional)
  bool corr = false;
  DescP dp{};
  const float *c_mean = nullptr, *c_inv_std = nullptr, *c_b2 = nullptr, *c_b3 = nullptr;
  const void* c_w5[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float c_scale = 1.f;
  void* c_X = nullptr;
  float* c_V = nullptr;
  float* c_F = nullptr;
  int32_t* c_status = nullptr;
  int c_stride = 1;          // refresh the correction every c_stride force evaluations (it is held in between)
  float last_corr_ms = 0.f;
};

namespace {

struct Layout {
  size_t off[64];
  int k = 0;
  size_t total = 0;
  size_t add(size_t bytes) {
    off[k] = total;
    total += a256(bytes);
    return k++;
  }
};

// Interleave the low 10 bits of three coordinates (z fastest): the Morton (Z-order) key of a cell.
uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
uint32_t morton3(uint32_t a, uint32_t b, uint32_t c) { return (spread10(a) << 2) | (spread10(b) << 1) | spread10(c); }

int tpa_of(const acs_engine_config* cfg) {
  const int t = cfg->tpa;
  return (t == 1 || t == 2 || t == 4 || t == 8 || t == 16 || t == 32) ? t : (t == 0 ? 1 : -1);
}

void plan(const acs_engine_config* cfg, std::vector<RepDev>& reps, std::vector<int64_t>& src0, int64_t& S, int32_t& T,
          int32_t& C, int32_t& NCH, int32_t& NCC, int& err) {
  const int tpa = tpa_of(cfg);
  if (tpa < 0) {
    err = ACS_ERR_ARG;
    return;
  }
  const int G = 32 / tpa;
  err = ACS_OK;
  if (cfg->cell_order != 0 && cfg->cell_order != 1) {
    err = ACS_ERR_ARG;
    return;
  }
  if (!(cfg->cell_scale == 0.0 || (cfg->cell_scale >= 1.0 && cfg->cell_scale <= 8.0))) {
    err = ACS_ERR_ARG;
    return;
  }
  const double cell_scale = cfg->cell_scale == 0.0 ? 1.0 : cfg->cell_scale;
  if (cfg->thermo.kind < 0 || cfg->thermo.kind > 2 ||
      (cfg->thermo.kind == 1 && !(cfg->thermo.kT >= 0.0 && cfg->thermo.friction >= 0.0)) ||
      (cfg->thermo.kind == 2 && !(cfg->thermo.kT > 0.0 && cfg->thermo.period > 0.0))) {
    err = ACS_ERR_ARG;
    return;
  }
  reps.clear();
  src0.clear();
  S = 0;
  T = 0;
  C = 0;
  NCH = 0;
  NCC = 0;
  int64_t g = 0;
  for (int r = 0; r < cfg->n_replicas; ++r) {
    const acs_replica& q = cfg->replicas[r];
    RepDev R{};
    if (q.n < 1 || !(q.rlist > 0.0) || !(q.half_skin >= 0.0) || !(q.dt > 0.0)) {
      err = ACS_ERR_ARG;
      return;
    }
    R.atom0 = S;
    R.n = q.n;
    R.npad = (q.n + 31) / 32 * 32;
    int64_t ncell = 1;
    bool small = false;   // list radius >= half a box edge
    for (int d = 0; d < 3; ++d) {
      if (!(q.box[d] > 0.0)) {
        err = ACS_ERR_ARG;
        return;
      }
      // cells no narrower than cell_scale x the list radius (so the 27-cell stencil is complete), at most
      // 1024 per edge
      double f = floor(q.box[d] / (q.rlist * cell_scale));
      int nc = f < 1.0 ? 1 : (int)std::min(f, 1024.0);
      while (nc > 1 && q.box[d] / nc < q.rlist) --nc;
      if (nc < 3) nc = 1;
      R.nc[d] = nc;
      R.L[d] = q.box[d];
      R.cs[d] = q.box[d] / nc;
      R.csf[d] = (float)R.cs[d];
      ncell *= nc;
      small |= q.rlist * 2.0 >= q.box[d];
    }
    if (err) return;
    R.cellbase = C;
    R.ncells = (int32_t)ncell;
    R.tile0 = (int32_t)(S / 32);
    R.ntiles = R.npad / 32;
    R.chunk0 = NCH;
    R.nchunks = (R.npad / G + kChunkTiles - 1) / kChunkTiles;
    R.cc0 = NCC;
    R.ncc = (int32_t)((ncell + kCellChunk - 1) / kCellChunk);
    NCC += R.ncc;
    R.dt = q.dt;
    R.hdt = 0.5 * q.dt;
    // A list entry keeps one periodic image per pair. When the list radius reaches half a box edge a pair's
    // minimum image can change between rebuilds, so such a replica rebuilds its lists every step (half skin 0:
    // every step flags it): each force evaluation then sees the minimum images of its own positions, as the
    // reference's per-evaluation re-imaging gives (accusim/forces.py:316-321).
    R.hs2 = small ? 0.0 : q.half_skin * q.half_skin;
    R.rl2 = q.rlist * q.rlist;
    if (cfg->thermo.kind == 2) {  // accusim/integrators.py:86-92: N_f = dim (n - 1), Q = N_f kT tau^2
      const double nf = 3.0 * (double)std::max(q.n - 1, 1);
      R.nh_nfkT = nf * cfg->thermo.kT;
      R.nh_Q = nf * cfg->thermo.kT * (cfg->thermo.period * cfg->thermo.period);
    }
    if (cfg->thermo.kind == 1) {  // accusim/integrators.py:65-66
      R.lv_c1 = exp(-cfg->thermo.friction * q.dt);
      for (int t = 0; t < cfg->ff.n_species && t < ACS_MAX_SPECIES; ++t)
        R.lv_sig[t] = sqrt((1.0 - R.lv_c1 * R.lv_c1) * cfg->thermo.kT / cfg->ff.mass[t]);
    }
    reps.push_back(R);
    src0.push_back(g);
    g += q.n;
    S += R.npad;
    C += (int32_t)ncell + 1;
    NCH += R.nchunks;
    T = (int32_t)(S / 32);
    if (S >= (int64_t)kIdxMask || C > INT32_MAX / 2 || (cfg->n_ex_ids > 0 && S >= (int64_t)kExBit)) {
      err = ACS_ERR_UNSUPPORTED;
      return;
    }
  }
  if (cfg->n_ex_ids < 0 || (cfg->n_ex_ids > 0 && (!cfg->ex_start || !cfg->ex_ids || cfg->ex_start[0] != 0))) {
    err = ACS_ERR_ARG;
    return;
  }
  for (int32_t a = 0; a < cfg->n_ex_ids; ++a) {
    if (cfg->ex_start[a + 1] < cfg->ex_start[a]) {
      err = ACS_ERR_ARG;
      return;
    }
  }
}

int32_t ex_count(const acs_engine_config* cfg) {
  return cfg->n_ex_ids > 0 && cfg->ex_start ? cfg->ex_start[cfg->n_ex_ids] : 0;
}

Layout make_layout(int32_t R, int64_t S, int32_t T, int32_t C, int32_t NCH, int32_t NCC, int32_t maxnb,
                   int32_t rec_cap, int64_t NG, int32_t n_ex_ids, int32_t n_ex) {
  Layout L;
  L.add(sizeof(RepDev) * R);                 // 0 rep
  L.add(4 * (size_t)R);                      // 1 active
  L.add(4 * (size_t)R);                      // 2 flag
  L.add(24 * (size_t)S);                     // 3 u
  L.add(24 * (size_t)S);                     // 4 v
  L.add(24 * (size_t)S);                     // 5 u0
  L.add(24 * (size_t)S);                     // 6 acc
  L.add(16 * (size_t)S);                     // 7 img0
  L.add(16 * (size_t)S);                     // 8 img1
  L.add(4 * (size_t)S);                      // 9 cellid
  L.add(4 * (size_t)S);                      // 10 id
  L.add(4 * (size_t)S);                      // 11 sp
  L.add(4 * (size_t)S * maxnb);              // 12 nbr
  L.add(4 * (size_t)S);                      // 13 nnb
  L.add(4 * (size_t)T);                      // 14 tile_rep
  L.add(4 * (size_t)C);                      // 15 cell_rep
  L.add(4 * (size_t)NCH);                    // 16 chunk_rep
  L.add(4 * (size_t)NCH);                    // 17 chunk_tile0
  L.add(4 * (size_t)NCH);                    // 18 chunk_ntiles
  L.add(24 * (size_t)S);                     // 19 xa
  L.add(24 * (size_t)S);                     // 20 tmp_xa
  L.add(24 * (size_t)S);                     // 21 tmp_v
  L.add(4 * (size_t)S);                      // 22 tmp_cell
  L.add(4 * (size_t)S);                      // 23 tmp_id
  L.add(4 * (size_t)S);                      // 24 tmp_sp
  L.add(4 * (size_t)S);                      // 25 newcell
  L.add(4 * (size_t)S);                      // 26 perm
  L.add(4 * (size_t)C);                      // 27 count
  L.add(4 * (size_t)C);                      // 28 start
  L.add(4 * (size_t)C);                      // 29 cursor
  L.add(8 * (size_t)NG * kRecW);             // 30 partials (one row per atom group)
  L.add(8 * (size_t)NCH * kRecW);            // 31 chunk partials
  L.add(8 * (size_t)rec_cap * R * kRecW);    // 32 records
  L.add(sizeof(acs_dev_status));             // 33 status
  L.add(16);                                 // 34 barrier
  L.add(8 * (size_t)R);                      // 35 src0
  L.add(4 * (size_t)NCC);                    // 36 cc_rep
  L.add(4 * (size_t)NCC);                    // 37 cc_c0
  L.add(4 * (size_t)NCC);                    // 38 cc_n
  L.add(4 * (size_t)NCC);                    // 39 cc_sum
  L.add(8 * 16);                             // 40 phase timers
  L.add(4 * (size_t)S);                      // 41 perm2
  L.add(8);                                  // 42 Langevin O-step counter
  L.add(8 * (size_t)NG);                     // 43 Nose-Hoover group partials
  L.add(8 * (size_t)NCH);                    // 44 Nose-Hoover chunk partials
  L.add(8 * 8 * (size_t)R);                  // 45 Nose-Hoover state
  L.add(8 * (size_t)rec_cap * R);            // 46 bath-energy records
  L.add(4 * ((size_t)R + 2));                // 47 flagged-cell prefix of a rebuild, list-build cell counter
  L.add(4 * ((size_t)n_ex_ids + 1));         // 48 DSF exclusions: CSR starts by atom id
  L.add(4 * ((size_t)n_ex + 1));             // 49 DSF exclusions: excluded ids
  L.add(4 * (size_t)C);                      // 50 crank (cell id -> slot-order position)
  L.add(4 * (size_t)C);                      // 51 cell_at (position -> cell id)
  L.add(4 * ((size_t)R + 2));                // 52 flagged one-cell-axis atoms prefix, list-build unit counter
  L.add(4 * ((size_t)T + 1));                // 53 flagged tiles of a rebuild and their count
  return L;
}

// erfc_as (the FP32 DSF pair term's Abramowitz & Stegun 7.1.26 erfc) evaluated in FP64 on the host with the same
// coefficients. The DSF shift constants come from it, so the engine's shifted potential and force vanish at rc
// under the approximation the pair term uses (with the exact erfc there they would jump by up to 1.5e-7 q_i q_j k
// / rc when a pair crosses the cutoff).
double erfc_as_host(double x) {
  const double t = 1.0 / fma(0.3275911, x, 1.0);
  const double q = fma(t, fma(t, fma(t, fma(t, 1.061405429, -1.453152027), 1.421413741), -0.284496736), 0.254829592);
  return t * q * exp(-x * x);
}

FFDev make_ff(const acs_forcefield& f, int& err) {
  FFDev ff{};
  err = ACS_OK;
  if (f.n_species < 1 || f.n_species > ACS_MAX_SPECIES || (!f.lj && !f.dsf)) {
    err = ACS_ERR_ARG;
    return ff;
  }
  const int S = ACS_MAX_SPECIES;
  ff.ns = f.n_species;
  ff.lj = f.lj;
  ff.dsf = f.dsf;
  for (int a = 0; a < f.n_species; ++a) {
    if (!(f.mass[a] > 0.0)) err = ACS_ERR_ARG;
    ff.mass[a] = f.mass[a];
    ff.inv_mass[a] = 1.0 / f.mass[a];
  }
  const double c6 = 1.0 / (f.lj_cutoff * f.lj_cutoff);
  const double src6 = c6 * c6 * c6;
  for (int a = 0; a < f.n_species; ++a)
    for (int b = 0; b < f.n_species; ++b) {
      const int p = a * S + b, q = a * f.n_species + b;
      const double e = f.lj ? f.lj_eps[q] : 0.0, s = f.lj ? f.lj_sig[q] : 1.0;
      ff.lj_eps4[p] = (float)(4.0 * e);
      ff.lj_eps24[p] = (float)(24.0 * e);
      ff.lj_sig2[p] = (float)(s * s);
      const double s6 = (s * s) * (s * s) * (s * s);
      ff.lj_a[p] = (float)(48.0 * e * s6 * s6);
      ff.lj_b[p] = (float)(24.0 * e * s6);
      ff.lj_c[p] = (float)(4.0 * e * s6 * s6);
      ff.lj_d[p] = (float)(4.0 * e * s6);
      ff.lj_rc2[p] = e > 0.0 ? (float)((f.lj_cutoff * s) * (f.lj_cutoff * s)) : 0.f;
      ff.lj_ushift[p] = (float)(4.0 * e * (src6 * src6 - src6));
      ff.qqk[p] = f.dsf ? (float)(f.dsf_k * f.q[a] * f.q[b]) : 0.f;
    }
  if (f.dsf) {
    const double a = f.dsf_alpha, rc = f.dsf_rcut;
    const double c = 2.0 * a / sqrt(M_PI);
    const double erc = erfc_as_host(a * rc);
    const double fshift = erc / (rc * rc) + c * exp(-(a * rc) * (a * rc)) / rc;
    ff.dsf_a = (float)a;
    ff.dsf_rc = (float)rc;
    ff.dsf_rc2 = (float)(rc * rc);
    ff.dsf_c = (float)c;
    ff.dsf_erc_rc = (float)(erc / rc);
    ff.dsf_fshift = (float)fshift;
    for (int s = 0; s < f.n_species; ++s) ff.self_e[s] = f.dsf_k * f.q[s] * f.q[s] * (erc / (2.0 * rc) + a / sqrt(M_PI));
  }
  return ff;
}

template <bool LJ, bool DSF, bool ONE>
int launch_step_t(acs_engine* e, int rec, int mode, int src, int dst, unsigned ostep, cudaStream_t s) {
  dim3 g(e->step_blocks), b(e->step_threads);
  const int th = e->E.thermo;
  if (mode == 0) {
    if (th == 1) {
      if (rec) k_step<LJ, DSF, true, 0, ONE, 1><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
      else k_step<LJ, DSF, false, 0, ONE, 1><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
    } else if (th == 2) {
      if (rec) k_step<LJ, DSF, true, 0, ONE, 2><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
      else k_step<LJ, DSF, false, 0, ONE, 2><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
    } else {
      if (rec) k_step<LJ, DSF, true, 0, ONE><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
      else if (e->pipe) k_step<LJ, DSF, false, 0, ONE, 0, true><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
      else k_step<LJ, DSF, false, 0, ONE><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
    }
  } else if (mode == 1) {
    if (th == 2) {
      if (rec) k_step<LJ, DSF, true, 1, ONE, 2><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
      else k_step<LJ, DSF, false, 1, ONE, 2><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
    } else {
      if (rec) k_step<LJ, DSF, true, 1, ONE><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
      else k_step<LJ, DSF, false, 1, ONE><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
    }
  } else {
    if (th == 2) k_step<LJ, DSF, true, 2, ONE, 2><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
    else k_step<LJ, DSF, true, 2, ONE><<<g, b, 0, s>>>(e->E, e->ff, src, dst, ostep);
  }
  return launch_status();
}

// Nose-Hoover after a step kernel (or at set-up): chunk sums of m v^2, the thermostat scalars (mode as in
// k_nh_scalars) and, after a step (modes 2, 3), the per-atom scale, for mode 3 with the next kick and drift.
int launch_nh(acs_engine* e, int mode, int rec, int rec_idx, int dst, cudaStream_t s) {
  if (e->E.thermo != 2) return ACS_OK;
  if (mode != 1) k_nh_chunks<<<(e->E.nchunks_total + 255) / 256, 256, 0, s>>>(e->E);
  k_nh_scalars<<<(e->E.R + 63) / 64, 64, 0, s>>>(e->E, mode, rec, rec_idx);
  if (mode == 2 || mode == 3) k_nh_apply<<<e->step_blocks, 256, 0, s>>>(e->E, mode == 3 ? 1 : 0, dst);
  return launch_status();
}

// ostep: offset of the O-step this launch's BAOAB takes, from the counter's value at the block start.
int launch_step(acs_engine* e, int rec, int mode, int src, int dst, unsigned ostep, cudaStream_t s) {
  const bool one = e->ff.ns == 1;
  if (e->ff.lj && e->ff.dsf)
    return one ? launch_step_t<true, true, true>(e, rec, mode, src, dst, ostep, s)
               : launch_step_t<true, true, false>(e, rec, mode, src, dst, ostep, s);
  if (e->ff.lj)
    return one ? launch_step_t<true, false, true>(e, rec, mode, src, dst, ostep, s)
               : launch_step_t<true, false, false>(e, rec, mode, src, dst, ostep, s);
  return one ? launch_step_t<false, true, true>(e, rec, mode, src, dst, ostep, s)
             : launch_step_t<false, true, false>(e, rec, mode, src, dst, ostep, s);
}

// Descriptors + tensor-core MLP -> per-slot correction forces for the images in buffer `src`.
int launch_correction(acs_engine* e, int src, cudaStream_t s) {
  if (!e->corr) return ACS_OK;
  const int64_t threads = e->E.S * 32;
  k_desc_engine<<<(int)((threads + 255) / 256), 256, 0, s>>>(e->E, src, e->dp, e->c_mean, e->c_inv_std,
                                                              (__nv_bfloat16*)e->c_X, e->c_V);
  int st = launch_status();
  if (st) return st;
  return acs_mlp_forward(e->c_X, e->c_V, e->E.S, e->c_w5, e->c_b2, e->c_b3, e->c_scale, e->c_F, e->c_status, s);
}

int launch_rebuild(acs_engine* e, int dst, int rec, int rec_idx, int force_all, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(e->coop_blocks);
  cfg.blockDim = dim3(256);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t err = e->E.ex_bit ? cudaLaunchKernelEx(&cfg, k_rebuild<true>, e->E, dst, rec, rec_idx, force_all)
                                 : cudaLaunchKernelEx(&cfg, k_rebuild<false>, e->E, dst, rec, rec_idx, force_all);
  return err == cudaSuccess ? ACS_OK : ACS_ERR_CUDA;
}

// A block of `steps` steps: prologue, rebuild check, then (step, rebuild check) x steps; records at the
// steps whose bit is set in rec_mask (bit k = step k of the block, 0-based); the last step stores the
// accelerations. Image buffers alternate 0,1.
int enqueue_block(acs_engine* e, int steps, const std::vector<char>& rec_at, cudaStream_t s) {
  int st = ACS_OK;
  if ((st = launch_nh(e, 1, 0, 0, 0, s))) return st;   // Nose-Hoover start half of the block's first step
  k_prologue<<<e->step_blocks, 256, 0, s>>>(e->E, 0);
  if ((st = launch_status())) return st;
  if ((st = launch_rebuild(e, 0, 0, 0, 0, s))) return st;
  int rec_idx = 0;
  for (int k = 0; k < steps; ++k) {
    const int src = k & 1, dst = (k + 1) & 1;
    const bool last = (k == steps - 1);
    const int rec = rec_at[k] ? 1 : 0;
    if (k % e->c_stride == 0 && (st = launch_correction(e, src, s))) return st;
    if ((st = launch_step(e, rec, last ? 1 : 0, src, dst, (unsigned)(k + 1), s))) return st;
    if ((st = launch_nh(e, last ? 2 : 3, rec, rec_idx, dst, s))) return st;
    if (!last || rec) {
      if ((st = launch_rebuild(e, dst, rec, rec_idx, 0, s))) return st;
    }
    rec_idx += rec;
  }
  if (e->E.thermo) {
    k_octr_advance<<<1, 1, 0, s>>>(e->E.octr, steps);
    return launch_status();
  }
  return ACS_OK;
}

}  // namespace

extern "C" {

size_t acs_engine_bytes(const acs_engine_config* cfg) {
  if (!cfg || cfg->n_replicas < 1 || cfg->n_replicas > kMaxRep || !cfg->replicas || cfg->maxnb < 1) return 0;
  std::vector<RepDev> reps;
  std::vector<int64_t> src0;
  int64_t S;
  int32_t T, C, NCH, NCC;
  int err;
  plan(cfg, reps, src0, S, T, C, NCH, NCC, err);
  if (err) return 0;
  return make_layout(cfg->n_replicas, S, T, C, NCH, NCC, cfg->maxnb, std::max(cfg->rec_cap, 1),
                     S / (32 / tpa_of(cfg)), cfg->n_ex_ids, ex_count(cfg)).total;
}

int acs_engine_create(const acs_engine_config* cfg, void* mem, size_t bytes, acs_engine** out) {
  if (!cfg || !out || !mem || cfg->n_replicas < 1 || cfg->n_replicas > kMaxRep || !cfg->replicas || cfg->maxnb < 1 ||
      cfg->maxnb > 4096)
    return ACS_ERR_ARG;
  if ((uintptr_t)mem & 255) return ACS_ERR_ARG;
  acs_engine* e = new acs_engine();
  int64_t S;
  int32_t T, C, NCH, NCC;
  int err;
  plan(cfg, e->reps, e->src0, S, T, C, NCH, NCC, err);
  if (err) {
    delete e;
    return err;
  }
  e->ff = make_ff(cfg->ff, err);
  if (err) {
    delete e;
    return err;
  }
  const int rec_cap = std::max(cfg->rec_cap, 1);
  const int tpa = tpa_of(cfg);
  const int G = 32 / tpa;
  Layout L = make_layout(cfg->n_replicas, S, T, C, NCH, NCC, cfg->maxnb, rec_cap, S / G, cfg->n_ex_ids,
                         ex_count(cfg));
  if (bytes < L.total) {
    delete e;
    return ACS_ERR_WORKSPACE;
  }
  char* b = (char*)mem;
  Eng& E = e->E;
  E.R = cfg->n_replicas;
  E.maxnb = cfg->maxnb;
  E.S = S;
  E.T = T;
  E.C = C;
  E.nchunks_total = NCH;
  E.tpa = tpa;
  E.G = G;
  E.NG = (int32_t)(S / G);
  E.rec_cap = rec_cap;
  E.rep = (RepDev*)(b + L.off[0]);
  E.active = (int32_t*)(b + L.off[1]);
  E.flag = (int32_t*)(b + L.off[2]);
  E.u = (double*)(b + L.off[3]);
  E.v = (double*)(b + L.off[4]);
  E.u0 = (double*)(b + L.off[5]);
  E.acc = (double*)(b + L.off[6]);
  E.img[0] = (float4*)(b + L.off[7]);
  E.img[1] = (float4*)(b + L.off[8]);
  E.cellid = (int32_t*)(b + L.off[9]);
  E.id = (int32_t*)(b + L.off[10]);
  E.sp = (int32_t*)(b + L.off[11]);
  E.nbr = (int32_t*)(b + L.off[12]);
  E.nnb = (int32_t*)(b + L.off[13]);
  E.tile_rep = (int32_t*)(b + L.off[14]);
  E.cell_rep = (int32_t*)(b + L.off[15]);
  E.chunk_rep = (int32_t*)(b + L.off[16]);
  E.chunk_tile0 = (int32_t*)(b + L.off[17]);
  E.chunk_ntiles = (int32_t*)(b + L.off[18]);
  E.xa = (double*)(b + L.off[19]);
  E.tmp_xa = (double*)(b + L.off[20]);
  E.tmp_v = (double*)(b + L.off[21]);
  E.tmp_cell = (int32_t*)(b + L.off[22]);
  E.tmp_id = (int32_t*)(b + L.off[23]);
  E.tmp_sp = (int32_t*)(b + L.off[24]);
  E.newcell = (int32_t*)(b + L.off[25]);
  E.perm = (int32_t*)(b + L.off[26]);
  E.count = (int32_t*)(b + L.off[27]);
  E.start = (int32_t*)(b + L.off[28]);
  E.cursor = (int32_t*)(b + L.off[29]);
  E.partials = (double*)(b + L.off[30]);
  E.chunk_part = (double*)(b + L.off[31]);
  E.rec = (double*)(b + L.off[32]);
  E.status = (acs_dev_status*)(b + L.off[33]);
  E.bar = (unsigned int*)(b + L.off[34]);
  e->src0_dev = (int64_t*)(b + L.off[35]);
  E.ncc = NCC;
  E.cc_rep = (int32_t*)(b + L.off[36]);
  E.cc_c0 = (int32_t*)(b + L.off[37]);
  E.cc_n = (int32_t*)(b + L.off[38]);
  E.cc_sum = (int32_t*)(b + L.off[39]);
  E.phase_ns = (unsigned long long*)(b + L.off[40]);
  E.perm2 = (int32_t*)(b + L.off[41]);
  E.octr = (unsigned long long*)(b + L.off[42]);
  E.nh_part = (double*)(b + L.off[43]);
  E.nh_chunk = (double*)(b + L.off[44]);
  E.nh_st = (double*)(b + L.off[45]);
  E.rec_bath = (double*)(b + L.off[46]);
  E.fcell = (int32_t*)(b + L.off[47]);
  E.n_ex_ids = cfg->n_ex_ids;
  E.ex_start = (const int32_t*)(b + L.off[48]);
  E.ex_ids = (const int32_t*)(b + L.off[49]);
  E.crank = (int32_t*)(b + L.off[50]);
  E.cell_at = (int32_t*)(b + L.off[51]);
  E.fsmall = (int32_t*)(b + L.off[52]);
  E.ftile = (int32_t*)(b + L.off[53]);
  E.ex_bit = cfg->n_ex_ids > 0 ? kExBit : 0u;
  E.jmask = cfg->n_ex_ids > 0 ? kExBit - 1u : kIdxMask;
  E.thermo = cfg->thermo.kind;
  E.spin_limit = cfg->barrier_wait_limit == 0 ? kSpinLimit : (cfg->barrier_wait_limit < 0 ? 0 : cfg->barrier_wait_limit);
  E.seed_lo = (uint32_t)cfg->thermo.seed;
  E.seed_hi = (uint32_t)(cfg->thermo.seed >> 32);

  // host-built index tables
  std::vector<int32_t> tile_rep(T), cell_rep(C), chunk_rep(NCH), chunk_t0(NCH), chunk_nt(NCH);
  std::vector<int32_t> cc_rep(NCC), cc_c0(NCC), cc_n(NCC);
  std::vector<int32_t> crank(C), cell_at(C);
  for (int r = 0; r < E.R; ++r) {
    const RepDev& R = e->reps[r];
    // slot order of the replica's cells: row-major (cell_order 0), or Morton (Z) order of the cell coordinates
    // (cell_order 1), which keeps the cells of one block of slots, and so their 27-cell neighbourhoods, compact
    std::vector<int32_t> order(R.ncells);
    for (int c = 0; c < R.ncells; ++c) order[c] = c;
    if (cfg->cell_order == 1) {
      std::vector<uint32_t> key(R.ncells);
      for (int c = 0; c < R.ncells; ++c) {
        const int c2 = c % R.nc[2], c1 = (c / R.nc[2]) % R.nc[1], c0 = c / (R.nc[2] * R.nc[1]);
        key[c] = morton3((uint32_t)c0, (uint32_t)c1, (uint32_t)c2);
      }
      std::stable_sort(order.begin(), order.end(), [&](int a, int b2) { return key[a] < key[b2]; });
    }
    for (int p = 0; p < R.ncells; ++p) {
      cell_at[R.cellbase + p] = R.cellbase + order[p];
      crank[R.cellbase + order[p]] = R.cellbase + p;
    }
    crank[R.cellbase + R.ncells] = cell_at[R.cellbase + R.ncells] = R.cellbase + R.ncells;   // sentinel
    for (int t = 0; t < R.ntiles; ++t) tile_rep[R.tile0 + t] = r;
    for (int c = 0; c <= R.ncells; ++c) cell_rep[R.cellbase + c] = r;
    for (int c = 0; c < R.ncc; ++c) {
      cc_rep[R.cc0 + c] = r;
      cc_c0[R.cc0 + c] = R.cellbase + c * kCellChunk;
      cc_n[R.cc0 + c] = std::min(kCellChunk, R.ncells - c * kCellChunk);
    }
    for (int c = 0; c < R.nchunks; ++c) {
      chunk_rep[R.chunk0 + c] = r;
      const int g0 = (int)(R.atom0 / G), ng = R.npad / G;
      chunk_t0[R.chunk0 + c] = g0 + c * kChunkTiles;
      chunk_nt[R.chunk0 + c] = std::min(kChunkTiles, ng - c * kChunkTiles);
    }
  }
  std::vector<int32_t> ones(E.R, 1), zeros(E.R, 0);
  acs_dev_status st0{};
  st0.fail_step = -1;
  unsigned int bar0[4] = {0, 0, 0, 0};
  bool ok = cudaGetDevice(&e->dev) == cudaSuccess;
  ok = ok && cudaMemcpy(E.rep, e->reps.data(), sizeof(RepDev) * E.R, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.active, ones.data(), 4 * E.R, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.flag, zeros.data(), 4 * E.R, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.tile_rep, tile_rep.data(), 4 * (size_t)T, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.cell_rep, cell_rep.data(), 4 * (size_t)C, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.chunk_rep, chunk_rep.data(), 4 * (size_t)NCH, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.chunk_tile0, chunk_t0.data(), 4 * (size_t)NCH, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.chunk_ntiles, chunk_nt.data(), 4 * (size_t)NCH, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.status, &st0, sizeof(st0), cudaMemcpyHostToDevice) == cudaSuccess;
  if (cfg->n_ex_ids > 0) {
    ok = ok && cudaMemcpy((void*)E.ex_start, cfg->ex_start, 4 * ((size_t)cfg->n_ex_ids + 1), cudaMemcpyHostToDevice) ==
                   cudaSuccess;
    const int32_t nnz = ex_count(cfg);
    if (nnz > 0)
      ok = ok && cudaMemcpy((void*)E.ex_ids, cfg->ex_ids, 4 * (size_t)nnz, cudaMemcpyHostToDevice) == cudaSuccess;
  }
  ok = ok && cudaMemcpy(E.bar, bar0, 16, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(e->src0_dev, e->src0.data(), 8 * (size_t)E.R, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.crank, crank.data(), 4 * (size_t)C, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.cell_at, cell_at.data(), 4 * (size_t)C, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.cc_rep, cc_rep.data(), 4 * (size_t)NCC, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.cc_c0, cc_c0.data(), 4 * (size_t)NCC, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(E.cc_n, cc_n.data(), 4 * (size_t)NCC, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemset(E.nnb, 0, 4 * (size_t)S) == cudaSuccess;
  ok = ok && cudaMemset(E.phase_ns, 0, 8 * 16) == cudaSuccess;
  ok = ok && cudaMemset(E.octr, 0, 8) == cudaSuccess;
  ok = ok && cudaMemset(E.nh_st, 0, 8 * 8 * (size_t)E.R) == cudaSuccess;
  ok = ok && cudaMemset(E.rec_bath, 0, 8 * (size_t)E.rec_cap * E.R) == cudaSuccess;
  int sms = 0, per_sm = 0;
  ok = ok && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->dev) == cudaSuccess;
  ok = ok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, E.ex_bit ? k_rebuild<true> : k_rebuild<false>,
                                                           256, 0) == cudaSuccess;
  if (!ok || per_sm < 1) {
    delete e;
    return ACS_ERR_CUDA;
  }
  // rebuild grid: at most 4 blocks per SM, and no more blocks than the largest phase can use (the list build
  // takes a warp per cell, or a warp per slot at >= 8 threads per atom; the other phases a thread per slot),
  // since each of its grid barriers costs in proportion to the blocks (small systems)
  const int64_t list_warps = tpa >= 8 ? S : (int64_t)C;
  const int64_t useful = std::max<int64_t>((S + 255) / 256, (list_warps + 7) / 8);
  e->coop_blocks = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * std::min(per_sm, 4), useful));
  const int grid_mult = cfg->grid_mult > 0 ? cfg->grid_mult : 0;
  // 128-thread step blocks when a 256-thread grid would fill fewer than two waves (4 blocks per SM): the
  // blocks then spread more evenly over the SMs (4096-ion NaCl: step kernel 6% faster; at 1M atoms 256 is
  // 0.3% faster)
  const int64_t need256 = (S / G * 32 + 255) / 256;
  e->step_threads = need256 < 2 * 4 * (int64_t)sms ? 128 : 256;
  const int64_t need = (S / G * 32 + e->step_threads - 1) / e->step_threads;
  e->step_blocks = (int)(grid_mult ? std::min<int64_t>(need, (int64_t)sms * grid_mult) : need);
  if (e->step_blocks < 1) e->step_blocks = 1;
  // under half a wave (16 warps per SM; the step kernel holds 32 at its 64 registers) the grid, not the registers,
  // sets the occupancy: the plain steps then take the variant with deeper load pipelining (up to 112 registers,
  // 16 warps per SM, so still one wave)
  e->pipe = (int64_t)e->step_blocks * e->step_threads / 32 <= 16 * (int64_t)sms;
  *out = e;
  return ACS_OK;
}

int acs_engine_set_state(acs_engine* e, const double* pos, const double* vel, const int32_t* species, void* stream) {
  if (!e || !pos || !vel || !species) return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  k_load<<<e->step_blocks, 256, 0, s>>>(e->E, pos, vel, species, e->src0_dev);
  int st = launch_status();
  if (st) return st;
  // build lists for every replica, then one force evaluation (accelerations + initial records)
  if ((st = launch_rebuild(e, 0, 0, 0, 1, s))) return st;
  if ((st = launch_correction(e, 0, s))) return st;
  if ((st = launch_step(e, 1, 2, 0, 0, 0u, s))) return st;
  if ((st = launch_nh(e, 0, 1, 0, 0, s))) return st;
  return launch_rebuild(e, 0, 1, 0, 0, s);
}

int acs_engine_get_state(acs_engine* e, double* pos, double* vel, double* acc, void* stream) {
  if (!e) return ACS_ERR_ARG;
  k_store<<<e->step_blocks, 256, 0, (cudaStream_t)stream>>>(e->E, pos, vel, acc, e->src0_dev);
  return launch_status();
}

int acs_engine_set_active(acs_engine* e, const int32_t* active_host, void* stream) {
  if (!e || !active_host) return ACS_ERR_ARG;
  return cudaMemcpyAsync(e->E.active, active_host, 4 * (size_t)e->E.R, cudaMemcpyHostToDevice, (cudaStream_t)stream) ==
                 cudaSuccess ? ACS_OK : ACS_ERR_CUDA;
}

int acs_engine_run(acs_engine* e, int32_t steps, int32_t record_every, int32_t record_last, void* stream) {
  if (!e || steps < 1 || record_every < 0) return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<char> rec_at(steps, 0);
  int nrec = 0;
  for (int k = 0; k < steps; ++k) {
    rec_at[k] = (record_every > 0 && (k + 1) % record_every == 0) || (record_last && k == steps - 1);
    nrec += rec_at[k];
  }
  if (nrec > e->E.rec_cap) return ACS_ERR_ARG;
  long long key = ((long long)steps << 32) ^ ((long long)record_every << 1) ^ (record_last ? 1 : 0);
  auto it = e->graphs.find(key);
  cudaGraphExec_t exec = nullptr;
  if (it == e->graphs.end()) {
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return ACS_ERR_CUDA;
    cudaGraph_t g = nullptr;
    int st = ACS_OK;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) st = ACS_ERR_CUDA;
    if (!st) st = enqueue_block(e, steps, rec_at, cs);
    cudaError_t ce = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (st || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return st ? st : ACS_ERR_CUDA;
    }
    if (cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
      cudaGraphDestroy(g);
      return ACS_ERR_CUDA;
    }
    cudaGraphDestroy(g);
    if (e->graphs.size() > 16) {
      for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
      e->graphs.clear();
    }
    e->graphs[key] = exec;
  } else {
    exec = it->second;
  }
  return cudaGraphLaunch(exec, s) == cudaSuccess ? ACS_OK : ACS_ERR_CUDA;
}

int acs_engine_records(acs_engine* e, double* out, int32_t count, void* stream) {
  if (!e || !out || count < 0 || count > e->E.rec_cap) return ACS_ERR_ARG;
  if (count == 0) return ACS_OK;
  return cudaMemcpyAsync(out, e->E.rec, 8 * (size_t)count * e->E.R * kRecW, cudaMemcpyDeviceToDevice,
                         (cudaStream_t)stream) == cudaSuccess ? ACS_OK : ACS_ERR_CUDA;
}

int acs_engine_status(acs_engine* e, acs_dev_status* out, int clear, void* stream) {
  if (!e || !out) return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(out, e->E.status, sizeof(acs_dev_status), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return ACS_ERR_CUDA;
  if (clear) {
    acs_dev_status z{};
    z.fail_step = -1;
    z.rebuilds = out->rebuilds;
    if (cudaMemcpyAsync(e->E.status, &z, sizeof(z), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return ACS_ERR_CUDA;
    // a barrier that timed out leaves its arrival count behind: start the next launch from a clean barrier
    if ((out->flags & ACS_FLAG_TIMEOUT) &&
        (cudaMemsetAsync(e->E.bar, 0, 16, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess))
      return ACS_ERR_CUDA;
  }
  return ACS_OK;
}

int acs_engine_neighbor_stats(acs_engine* e, int32_t* max_nnb, int64_t* sum_nnb, void* stream) {
  if (!e) return ACS_ERR_ARG;
  std::vector<int32_t> h(e->E.S);
  if (cudaMemcpyAsync(h.data(), e->E.nnb, 4 * (size_t)e->E.S, cudaMemcpyDeviceToHost, (cudaStream_t)stream) !=
          cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return ACS_ERR_CUDA;
  int32_t mx = 0;
  int64_t sm = 0;
  for (int32_t v : h) {
    mx = std::max(mx, v);
    sm += v;
  }
  if (max_nnb) *max_nnb = mx;
  if (sum_nnb) *sum_nnb = sm;
  return ACS_OK;
}

int acs_engine_launch_info(acs_engine* e, int32_t* step_blocks, int32_t* coop_blocks, int64_t* slots) {
  if (!e) return ACS_ERR_ARG;
  if (step_blocks) *step_blocks = e->step_blocks;
  if (coop_blocks) *coop_blocks = e->coop_blocks;
  if (slots) *slots = e->E.S;
  return ACS_OK;
}

int acs_engine_load_state(acs_engine* e, const double* pos, const double* vel, void* stream) {
  if (!e || !pos || !vel) return ACS_ERR_ARG;
  k_load_keep<<<e->step_blocks, 256, 0, (cudaStream_t)stream>>>(e->E, pos, vel, e->src0_dev);
  int st = launch_status();
  if (st || e->E.thermo != 2) return st;
  // new velocities: the next start half needs their kinetic-energy sum
  k_nh_ke<<<(e->E.NG + 255) / 256, 256, 0, (cudaStream_t)stream>>>(e->E, e->ff);
  return launch_nh(e, 0, 0, 0, 0, (cudaStream_t)stream);
}

int acs_engine_count_pairs(acs_engine* e, unsigned long long* out_dev, void* stream) {
  if (!e || !out_dev) return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(out_dev, 0, 16, s) != cudaSuccess) return ACS_ERR_CUDA;
  // images of buffer 0 are current after acs_engine_set_state (and after any rebuild into buffer 0)
  k_count_pairs<<<e->step_blocks, 256, 0, s>>>(e->E, e->ff, 0, out_dev);
  return launch_status();
}

int acs_engine_dump_lists(acs_engine* e, long long* keys_dev, long long cap, unsigned long long* count_dev,
                          double* pos_build_dev, void* stream) {
  if (!e || !count_dev || cap < 0 || (cap > 0 && !keys_dev)) return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(count_dev, 0, sizeof(unsigned long long), s) != cudaSuccess) return ACS_ERR_CUDA;
  int64_t n_total = 0;
  for (const RepDev& R : e->reps) n_total += R.n;
  k_dump_lists<<<e->step_blocks, 256, 0, s>>>(e->E, e->src0_dev, n_total, keys_dev, cap, count_dev, pos_build_dev);
  return launch_status();
}

// The same launch sequence as one graph block, launched eagerly with CUDA events around every kernel, for
// per-kernel timing. out_ms[0] = total step-kernel ms, [1] = total list-maintenance ms, [2] = step launches,
// [3] = list-maintenance launches. Synchronous.
int acs_engine_run_timed(acs_engine* e, int32_t steps, int32_t record_every, float* out_ms, void* stream) {
  if (!e || steps < 1 || !out_ms) return ACS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<cudaEvent_t> ev(6 * (size_t)steps + 4);
  for (auto& x : ev)
    if (cudaEventCreate(&x) != cudaSuccess) return ACS_ERR_CUDA;
  int st = ACS_OK;
  size_t ne = 0;
  std::vector<std::pair<size_t, int>> spans;  // (first event index, kind)
  auto mark = [&](int kind, auto&& launch) {
    cudaEventRecord(ev[ne], s);
    int r = launch();
    cudaEventRecord(ev[ne + 1], s);
    spans.push_back({ne, kind});
    ne += 2;
    return r;
  };
  st = launch_nh(e, 1, 0, 0, 0, s);
  if (!st) k_prologue<<<e->step_blocks, 256, 0, s>>>(e->E, 0);
  if (!st) st = launch_status();
  if (!st) st = launch_rebuild(e, 0, 0, 0, 0, s);
  int rec_idx = 0;
  for (int k = 0; k < steps && !st; ++k) {
    const int src = k & 1, dst = (k + 1) & 1;
    const bool last = (k == steps - 1);
    const int rec = ((record_every > 0 && (k + 1) % record_every == 0) || last) ? 1 : 0;
    if (e->corr && k % e->c_stride == 0) st = mark(2, [&] { return launch_correction(e, src, s); });
    if (!st) st = mark(0, [&] {
      int q = launch_step(e, rec, last ? 1 : 0, src, dst, (unsigned)(k + 1), s);
      return q ? q : launch_nh(e, last ? 2 : 3, rec, rec_idx < e->E.rec_cap ? rec_idx : 0, dst, s);
    });
    if (!st) st = mark(1, [&] { return launch_rebuild(e, dst, rec, rec_idx < e->E.rec_cap ? rec_idx : 0, 0, s); });
    rec_idx += rec;
  }
  if (!st && e->E.thermo) {
    k_octr_advance<<<1, 1, 0, s>>>(e->E.octr, steps);
    st = launch_status();
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) st = ACS_ERR_CUDA;
  float tot[3] = {0.f, 0.f, 0.f};
  int cnt[3] = {0, 0, 0};
  for (auto& sp : spans) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev[sp.first], ev[sp.first + 1]) == cudaSuccess) {
      tot[sp.second] += ms;
      cnt[sp.second] += 1;
    }
  }
  for (auto& x : ev) cudaEventDestroy(x);
  out_ms[0] = tot[0];
  out_ms[1] = tot[1];
  out_ms[2] = (float)cnt[0];
  out_ms[3] = (float)cnt[1];
  e->last_corr_ms = cnt[2] ? tot[2] / cnt[2] : 0.f;
  return st;
}

int acs_engine_phase_times(acs_engine* e, unsigned long long* out16, int clear) {
  if (!e || !out16) return ACS_ERR_ARG;
  if (cudaMemcpy(out16, e->E.phase_ns, 8 * 16, cudaMemcpyDeviceToHost) != cudaSuccess) return ACS_ERR_CUDA;
  if (clear && cudaMemset(e->E.phase_ns, 0, 8 * 16) != cudaSuccess) return ACS_ERR_CUDA;
  return ACS_OK;
}

int acs_engine_set_correction(acs_engine* e, const float* params6, const float* mean, const float* inv_std,
                              const void* const* w5, const float* b2, const float* b3, float out_scale, void* X,
                              float* V, float* F, int32_t* status_dev, int enabled) {
  if (!e) return ACS_ERR_ARG;
  if (enabled && (!params6 || !mean || !inv_std || !w5 || !b2 || !b3 || !X || !V || !F || !status_dev))
    return ACS_ERR_ARG;
  for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
  e->graphs.clear();
  e->corr = enabled != 0;
  e->E.fext = e->corr ? F : nullptr;
  if (!e->corr) return ACS_OK;
  e->dp.r0 = params6[0];
  e->dp.dmu = params6[1];
  e->dp.inv2s2 = params6[2];
  e->dp.rc2 = params6[3] * params6[3];
  e->dp.pi_rc = (float)M_PI / params6[3];
  e->c_mean = mean;
  e->c_inv_std = inv_std;
  for (int k = 0; k < 5; ++k) e->c_w5[k] = w5[k];
  e->c_b2 = b2;
  e->c_b3 = b3;
  e->c_scale = out_scale;
  e->c_X = X;
  e->c_V = V;
  e->c_F = F;
  e->c_status = status_dev;
  return ACS_OK;
}

float acs_engine_last_correction_ms(acs_engine* e) { return e ? e->last_corr_ms : 0.f; }

int acs_engine_nh_state(acs_engine* e, double* xi_eta, int32_t set) {
  if (!e || !xi_eta) return ACS_ERR_ARG;
  std::vector<double> st(8 * (size_t)e->E.R);
  if (cudaMemcpy(st.data(), e->E.nh_st, 8 * st.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return ACS_ERR_CUDA;
  for (int r = 0; r < e->E.R; ++r) {
    if (set) {
      st[8 * r] = xi_eta[2 * r];
      st[8 * r + 1] = xi_eta[2 * r + 1];
    } else {
      xi_eta[2 * r] = st[8 * r];
      xi_eta[2 * r + 1] = st[8 * r + 1];
    }
  }
  if (set && cudaMemcpy(e->E.nh_st, st.data(), 8 * st.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return ACS_ERR_CUDA;
  return ACS_OK;
}

int acs_engine_bath_records(acs_engine* e, double* out_dev, int32_t count, void* stream) {
  if (!e || !out_dev || count < 0 || count > e->E.rec_cap) return ACS_ERR_ARG;
  return cudaMemcpyAsync(out_dev, e->E.rec_bath, 8 * (size_t)count * e->E.R, cudaMemcpyDeviceToDevice,
                         (cudaStream_t)stream) == cudaSuccess ? ACS_OK : ACS_ERR_CUDA;
}

int acs_engine_set_correction_stride(acs_engine* e, int32_t stride) {
  if (!e || stride < 1) return ACS_ERR_ARG;
  if (stride != e->c_stride) {
    for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
    e->graphs.clear();
  }
  e->c_stride = stride;
  return ACS_OK;
}

int acs_engine_destroy(acs_engine* e) {
  if (!e) return ACS_OK;
  for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
  delete e;
  return ACS_OK;
}

}  // extern "C"
