/*
 * accusim_b200: C ABI of the B200 (sm_100a) short-range force-and-step library.
 *
 * Every entry point takes raw DEVICE pointers owned by the caller, plain sizes, and a CUDA stream
 * passed as `void*` (a cudaStream_t; NULL = legacy default stream). Calls never allocate device
 * memory (scratch is passed in as `work` with its byte size), never synchronise the device (except
 * the engine calls documented as synchronous), never throw, and return an acs_status. Kernel-side
 * conditions (list overflow, non-finite force, barrier timeout) are written to a caller-owned device
 * status block that the caller reads after its own synchronisation.
 *
 * Reference interfaces replaced (paths inside the accusim project, erezbz/DevinProj):
 *   acs_grid_* / acs_nlist_*     accusim/forces.py:279-321 cell_list_pairs, :78-98 VerletList.pairs
 *   acs_lj_fp64                  accusim/forces.py:119-175 LennardJones.compute (list and dense paths)
 *   acs_dsf_fp64                 accusim/forces.py:408-452 DampedShiftedCoulomb.compute
 *   acs_vv_*                     accusim/integrators.py:25-31 VelocityVerlet.step,
 *                                accusim/system.py:124-129 apply_boundaries, simulation.py:67-70
 *   acs_rdf_hist                 accusim/analysis.py:7-24 rdf (pair-distance histogram)
 *   acs_langevin_ou              accusim/integrators.py:50-71 Langevin.step (the O-step; B and A reuse acs_vv_*)
 *   acs_reduce_conserved         accusim/system.py:106-114 kinetic_energy / momentum / angular_momentum
 *   acs_engine_*                 accusim/simulation.py:95-112 Simulation.run driving VelocityVerlet with
 *                                LennardJones and/or DampedShiftedCoulomb (device-resident fast path)
 */
#ifndef ACCUSIM_B200_H
#define ACCUSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ACS_ABI_VERSION 1

typedef enum acs_status {
  ACS_OK = 0,
  ACS_ERR_ARG = 1,          /* bad argument (null pointer, size, alignment) */
  ACS_ERR_WORKSPACE = 2,    /* work buffer smaller than the *_work_bytes query */
  ACS_ERR_CUDA = 3,         /* a CUDA runtime call failed (launch, graph, attribute) */
  ACS_ERR_LIST_OVERFLOW = 4,/* neighbour list capacity exceeded: rebuild with the reported need */
  ACS_ERR_NONFINITE = 5,    /* NaN/Inf force or position */
  ACS_ERR_TIMEOUT = 6,      /* a bounded device-side barrier wait gave up */
  ACS_ERR_UNSUPPORTED = 7,  /* size or mode outside what the library supports */
  ACS_ERR_NO_DEVICE = 8
} acs_status;

/* Device status block written by kernels (caller zeroes it with acs_status_clear or a memset). */
typedef struct acs_dev_status {
  int32_t flags;       /* bit 0 list overflow, bit 1 non-finite, bit 2 barrier timeout */
  int32_t need_nbr;    /* largest neighbour count seen in a build (valid when overflow is set) */
  int32_t rebuilds;    /* engine: neighbour-list rebuilds performed */
  int32_t fail_step;   /* engine: first step index whose work was skipped after an error, or -1 */
  int32_t steps_done;  /* engine: steps completed */
  int32_t pad[3];
} acs_dev_status;

#define ACS_FLAG_OVERFLOW 1
#define ACS_FLAG_NONFINITE 2
#define ACS_FLAG_TIMEOUT 4

int acs_abi_version(void);
const char* acs_status_string(int status);
/* Number of SMs and compute capability of the current device (host query, no device memory). */
int acs_device_info(int* sm_count, int* cc_major, int* cc_minor);

/* ---------------------------------------------------------------- cell grid + neighbour list --
 * Binning of accusim/forces.py:283-291: periodic boxes bin over [0, box) with ncell = floor(box/rc)
 * (collapsed to 1 per dimension when < 3); open systems bin over [min, max] with span >= rc. The
 * host fills acs_grid (acs_grid_setup does it from the box and, for open systems, the position
 * bounds). The list holds, for every atom i, ALL j != i with minimum-image |d|^2 < rc^2, computed
 * with the reference's FP64 expression d -= box*round(d/box), r^2 = (dx^2 + dy^2) + dz^2 (IEEE
 * round-to-nearest, no FMA), so its pair set equals cell_list_pairs' up to r^2 ties within 1 ulp.
 * Layout: nbr[(i/32)*maxnb*32 + k*32 + i%32] = j (k-th neighbour of i), nnb[i] = count. */
typedef struct acs_grid {
  double lo[3];
  double span[3];
  double box[3];
  int32_t ncell[3];
  int32_t periodic;
  double rc;    /* list radius (cutoff + skin) */
  double rc2;   /* rc**2 as the host computes it */
} acs_grid;

/* Fill *g for a box (box3 may be NULL for an open system; then lo3/hi3 are the position bounds). */
int acs_grid_setup(acs_grid* g, const double* box3, int periodic, const double* lo3, const double* hi3, double rc);
size_t acs_nlist_work_bytes(int64_t n, const acs_grid* g);
int acs_nlist_build(const double* pos, int64_t n, const acs_grid* g, int32_t maxnb, int32_t* nbr, int32_t* nnb,
                    void* work, size_t work_bytes, acs_dev_status* status, void* stream);
/* Unique pairs i<j of a built list, written in row order of i; *count_dev receives the total.
 * Capacity `cap`; pairs beyond it are counted but not written. */
int acs_nlist_pairs(const int32_t* nbr, const int32_t* nnb, int64_t n, int32_t maxnb, int32_t* pi, int32_t* pj,
                    int64_t cap, unsigned long long* count_dev, void* stream);
/* Pair-distance histogram for the radial distribution function, replaces the O(n^2) pair loop of
 * accusim/analysis.py:7-24 (rdf): counts of pairs i < j (both of species `species`; all atoms when it is
 * negative) with minimum-image distance r <= rmax in `bins` equal bins of [0, rmax], r and the bin index
 * computed as the reference computes them (FP64 minimum image, sqrt, NumPy's uniform-bin histogram rule).
 * hist_dev: bins uint64 counts (device). g: a periodic grid from acs_grid_setup with rc >= rmax (the
 * caller normalises by the ideal-gas shell counts). bins <= 8192. Work from acs_rdf_work_bytes. */
size_t acs_rdf_work_bytes(int64_t n, const acs_grid* g);
int acs_rdf_hist(const double* pos, const int32_t* sp, int64_t n, const acs_grid* g, int32_t species, int32_t bins,
                 double rmax, unsigned long long* hist_dev, void* work, size_t work_bytes, void* stream);
/* Skin test of accusim/forces.py:88-94: flag_dev = 1 if max_i |x_i - x0_i|^2 (minimum image) >= half_skin2. */
int acs_nlist_displacement(const double* pos, const double* pos0, int64_t n, const double* box3, int periodic,
                           double half_skin2, int32_t* flag_dev, void* stream);

/* ---------------------------------------------------------------- FP64 drop-in forces --------
 * Forces in SI, FP64, each atom summing its own full neighbour list (no atomics, deterministic).
 * nbr == NULL selects the dense all-pairs path (accusim/forces.py:162-175, :439-452).
 * Species tables are n_species x n_species row-major FP64, host pointers (copied to the device).
 * energy_dev receives sum_i e_i (FP64, deterministic two-level reduction). */
size_t acs_force_work_bytes(int64_t n);
int acs_lj_fp64(const double* pos, const int32_t* sp, int64_t n, const double* box3, int periodic,
                const int32_t* nbr, const int32_t* nnb, int32_t maxnb, int32_t n_species, const double* eps_tab,
                const double* sig_tab, double cutoff, double* force, double* energy_dev, void* work,
                size_t work_bytes, void* stream);
/* acs_lj_fp64 for callers that cannot allocate device memory (their own pool owns the GPU, allocation is
 * forbidden after start-up, or the host hands out only input/output buffers). No counterpart in the
 * reference. Same arguments and results as acs_lj_fp64 without the work buffer: the reduction scratch is a
 * 64 KiB static device array inside the library, held on every GPU that loads it until exit, so
 * n <= 2,097,152 (ACS_ERR_UNSUPPORTED above). The first call in each CUDA context (a device's primary context,
 * or a context a driver-API caller made current) looks up that array's address in the context, so make it
 * before any stream capture. Calls share the array: calls that overlap on the GPU race. */
int acs_lj_fp64_noalloc(const double* pos, const int32_t* sp, int64_t n, const double* box3, int periodic,
                        const int32_t* nbr, const int32_t* nnb, int32_t maxnb, int32_t n_species,
                        const double* eps_tab, const double* sig_tab, double cutoff, double* force,
                        double* energy_dev, void* stream);
/* DSF: per-atom charges q (C), exclusions as CSR over atom indices (ex_start[n+1], ex_idx; may be NULL).
 * force/energy are returned multiplied by k, the self term included in energy_dev. */
int acs_dsf_fp64(const double* pos, const double* q, int64_t n, const double* box3, int periodic,
                 const int32_t* nbr, const int32_t* nnb, int32_t maxnb, const int32_t* ex_start,
                 const int32_t* ex_idx, double alpha, double rcut, double k, double* force, double* energy_dev,
                 void* work, size_t work_bytes, void* stream);

/* ---------------------------------------------------------------- FP64 VelocityVerlet ---------
 * Same IEEE operation order as accusim/integrators.py:27-31 and system.py:124-129 (no FMA), so a
 * step is bit-identical to the reference given bit-identical accelerations. */
int acs_vv_kick(double* vel, const double* acc, int64_t n, double half_dt, void* stream);
int acs_vv_drift_wrap(double* pos, const double* vel, int64_t n, double dt, const double* box3, int periodic,
                      void* stream);
/* Langevin BAOAB O-step, replaces accusim/integrators.py:65-67 (Langevin.step): vel = c1 * vel + sig[i] *
 * noise with c1 = exp(-gamma dt) and sig[i] = sqrt((1 - c1^2) kT / m_i) computed by the caller, noise the
 * caller's standard normal draws (n x 3). The half drifts around it are acs_vv_drift_wrap with dt / 2. */
int acs_langevin_ou(double* vel, const double* noise, const double* sig, int64_t n, double c1, void* stream);
/* acc = force / mass[species] (accusim/simulation.py:70). */
int acs_vv_accel(double* acc, const double* force, const int32_t* sp, const double* species_mass, int32_t n_species,
                 int64_t n, void* stream);
/* out_dev[0] = KE, [1..3] = P, [4..6] = L (accusim/system.py:106-114), FP64, deterministic. */
size_t acs_reduce_work_bytes(int64_t n);
int acs_reduce_conserved(const double* pos, const double* vel, const int32_t* sp, const double* species_mass,
                         int32_t n_species, int64_t n, double* out_dev, void* work, size_t work_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ACCUSIM_B200_H */
