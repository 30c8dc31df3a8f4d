/*
 * accusim_b200 engine: device-resident fast path for Simulation.run with VelocityVerlet and
 * LennardJones and/or DampedShiftedCoulomb (accusim/simulation.py:95-112, integrators.py:25-31,
 * forces.py:78-175, :391-452), for one periodic system or a batch of independent replicas.
 *
 * Arithmetic: FP64 positions (as offsets from cell origins) and velocities, FP64 integration and
 * conserved-quantity sums; FP32 pair terms with Kahan-compensated per-atom force and energy sums.
 * Units are the caller's (the Python layer uses A, u, kJ/mol, e). Memory: the caller allocates one
 * 256-byte-aligned device block of acs_engine_bytes() and passes it to acs_engine_create; the engine
 * keeps only host-side bookkeeping and cached CUDA graphs. Multi-step runs are CUDA graphs of
 * one fused force/kick/drift kernel and one cooperative list-maintenance kernel per step.
 */
#ifndef ACCUSIM_B200_ENGINE_H
#define ACCUSIM_B200_ENGINE_H

#include "accusim_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct acs_replica {
  int32_t n;          /* atoms */
  int32_t pad;
  double box[3];      /* periodic box edges */
  double dt;          /* time step */
  double rlist;       /* neighbour-list radius = largest cutoff + skin (>= half a box edge: lists rebuilt every step) */
  double half_skin;   /* rebuild once an atom has moved this far since the last build */
} acs_replica;

typedef struct acs_forcefield {
  int32_t n_species;  /* <= 8 */
  int32_t lj;         /* LennardJones term on */
  int32_t dsf;        /* DampedShiftedCoulomb term on */
  int32_t pad;
  double mass[8];
  double lj_eps[64];  /* n_species x n_species, mixed (Lorentz-Berthelot) */
  double lj_sig[64];
  double lj_cutoff;   /* in units of sigma_ij; energy shifted to zero there */
  double dsf_alpha, dsf_rcut, dsf_k;
  double q[8];        /* charge per species */
} acs_forcefield;

/* Thermostat of the engine's step. kind 0: VelocityVerlet (accusim/integrators.py:25-31); kind 1:
 * Langevin BAOAB (accusim/integrators.py:50-71) with c1 = exp(-friction dt) and sigma = sqrt((1 - c1^2)
 * kT / m) per species and replica. Its standard normal draws are counter-based (Philox4x32-10, key = seed,
 * counter = (O-step index, atom index within the replica, replica)), so a run is reproducible and does
 * not depend on list rebuilds or on which other replicas share the engine. kind 2: Nose-Hoover with the
 * Trotter half-steps of accusim/integrators.py:74-116, one thermostat per replica (N_f = 3 (n - 1),
 * Q = N_f kT period^2), its (xi, eta) read and set with acs_engine_nh_state. */
typedef struct acs_thermostat {
  int32_t kind;
  int32_t pad;
  double kT;          /* k_B T in the caller's energy unit */
  double friction;    /* Langevin gamma, in 1 / caller time unit */
  uint64_t seed;      /* Langevin draws */
  double period;      /* Nose-Hoover thermostat period, caller time unit */
} acs_thermostat;

typedef struct acs_engine_config {
  int32_t n_replicas;
  int32_t maxnb;      /* neighbour capacity per atom */
  int32_t rec_cap;    /* records kept per run call */
  int32_t grid_mult;  /* step kernel: blocks per SM (0 = one thread per atom slot) */
  int32_t tpa;        /* threads per atom in the pair kernel: 1, 2, 4, 8, 16 or 32 (0 = 1) */
  int32_t cell_order; /* slot order of the cells (atoms are sorted by cell at every rebuild): 0 row-major,
                       * 1 Morton (Z) order of the cell coordinates; results are deterministic either way */
  const acs_replica* replicas;  /* host array */
  acs_forcefield ff;
  acs_thermostat thermo;        /* zero: VelocityVerlet */
  /* DampedShiftedCoulomb exclusions (accusim/forces.py:400, 418-426: atom pairs with no DSF interaction;
   * the LJ term stays), the same for every replica, as host arrays in CSR form by atom index within a
   * replica (the caller's order): the atoms excluded for atom a are ex_ids[ex_start[a] .. ex_start[a + 1]),
   * listed from both sides. n_ex_ids = 0 (NULL arrays): none. With exclusions an engine holds fewer than
   * 2^26 atom slots. */
  const int32_t* ex_start;      /* n_ex_ids + 1 entries, ex_start[0] = 0, non-decreasing */
  const int32_t* ex_ids;        /* ex_start[n_ex_ids] entries */
  int32_t n_ex_ids;
  int32_t pad2;
  /* Grid-barrier waits of the cooperative list-maintenance kernel: a block polls up to this many times,
   * 100 ns apart, then reports ACS_FLAG_TIMEOUT (acs_engine_status; later kernels of the engine return at
   * once until the status is cleared, which also resets the barrier) and its kernel returns.
   * 0: the default, 2e7 polls (~2 s); negative: no polling (a block that is not the last to arrive gives up
   * at once, which makes the timeout path testable). */
  int64_t barrier_wait_limit;
  /* Cell edge of the list build, in units of the list radius: cells no narrower than cell_scale x rlist
   * (0: 1, the narrowest cells the 27-cell stencil covers; otherwise 1 <= cell_scale <= 8). Wider cells put
   * more home atoms in each cell a warp takes and more candidates in its stencil, and change the slot order;
   * the neighbour pair set is the same for every value (it is the FP64 filter's at the list radius). */
  double cell_scale;
} acs_engine_config;

typedef struct acs_engine acs_engine;

size_t acs_engine_bytes(const acs_engine_config* cfg);
int acs_engine_create(const acs_engine_config* cfg, void* mem, size_t bytes, acs_engine** out);
/* pos/vel: device, replica-concatenated (n_r x 3 each, caller units), species: device int32.
 * Builds every list, evaluates forces, and writes the initial records at index 0. */
int acs_engine_set_state(acs_engine* e, const double* pos, const double* vel, const int32_t* species, void* stream);
/* Device outputs in caller order; positions wrapped into [0, box) as accusim/system.py:127 does. */
int acs_engine_get_state(acs_engine* e, double* pos, double* vel, double* acc, void* stream);
/* Host array of n_replicas flags: inactive replicas are skipped by later runs. */
int acs_engine_set_active(acs_engine* e, const int32_t* active_host, void* stream);
/* Advance active replicas by `steps` (one cached CUDA graph per (steps, record schedule)). Records are
 * taken after steps k with (k+1) % record_every == 0 and, if record_last, after the last step; record i
 * of replica r is [KE, PE, Px, Py, Pz, Lx, Ly, Lz] at rec[(i * n_replicas + r) * 8]. */
int acs_engine_run(acs_engine* e, int32_t steps, int32_t record_every, int32_t record_last, void* stream);
int acs_engine_records(acs_engine* e, double* out_dev, int32_t count, void* stream);
/* Replace positions/velocities (device, caller order, wrapped or not) keeping the current lists and
 * accelerations; the next run's skin test rebuilds the lists if the new positions require it. */
int acs_engine_load_state(acs_engine* e, const double* pos, const double* vel, void* stream);
/* out_dev[0] = ordered LJ pairs inside cutoff*sigma_ij, out_dev[1] = ordered DSF pairs inside rc (each
 * unordered pair counted twice), on the images set by the last acs_engine_set_state. */
int acs_engine_count_pairs(acs_engine* e, unsigned long long* out_dev, void* stream);
/* The engine's neighbour lists as they are, for checking them against accusim's pair search
 * (accusim/forces.py:279-321 cell_list_pairs, accusim/forces.py:86-98 VerletList.pairs) at the list radius:
 * every list entry as a directed pair of caller indices (global over replicas, in replica order),
 * keys_dev[k] = 2 (i n_total + j) + excluded, excluded = the entry's DSF exclusion flag (-1 for an entry
 * that does not name an atom of its own replica), in no particular order; *count_dev = number of entries
 * (entries beyond cap are counted, not written). pos_build_dev (optional, n_total x 3) receives the FP64
 * absolute positions of the last rebuild, from which the lists were built. Device arrays. */
int acs_engine_dump_lists(acs_engine* e, long long* keys_dev, long long cap, unsigned long long* count_dev,
                          double* pos_build_dev, void* stream);
/* Synchronous: copies the device status block to *out (optionally clearing its error flags). */
int acs_engine_status(acs_engine* e, acs_dev_status* out, int clear, void* stream);
int acs_engine_neighbor_stats(acs_engine* e, int32_t* max_nnb, int64_t* sum_nnb, void* stream);
int acs_engine_launch_info(acs_engine* e, int32_t* step_blocks, int32_t* coop_blocks, int64_t* slots);
/* The launch sequence of one block, eager, with CUDA events around every kernel (synchronous):
 * out_ms = {step-kernel ms total, list-maintenance ms total, step launches, list-maintenance launches}. */
int acs_engine_run_timed(acs_engine* e, int32_t steps, int32_t record_every, float* out_ms, void* stream);
/* Accumulated wall time (ns, device global timer, block 0's view) of the list-maintenance phases:
 * [1] flag read, [2] clear, [3] bin, [4..6] scan, [7] scatter, [8] in-cell sort, [9] gather, [10] commit,
 * [15] list build (block 0 share). Synchronous. */
int acs_engine_phase_times(acs_engine* e, unsigned long long* out16, int clear);
/* Learned force correction (no counterpart in the reference): when enabled, every force evaluation first
 * computes the radial descriptors of all slots from the engine's images and lists (radius params6[3] <= list
 * radius) into X (S x 80 BF16) and V (S x 64 x 3 FP32), runs the tensor-core MLP (acs_mlp_forward) into
 * F (S x 3 FP32, slot order, engine force units) and adds F to the pair forces. Buffers are caller-owned
 * (S = acs_engine_launch_info's slots). Changing it drops the cached graphs. */
int acs_engine_set_correction(acs_engine* e, const float* params6, const float* mean, const float* inv_std,
                              const void* const* w5, const float* b2, const float* b3, float out_scale, void* X,
                              float* V, float* F, int32_t* status_dev, int enabled);
/* Refresh the correction every `stride` force evaluations of a block (the first of each block always) and
 * hold it in between (a multiple-time-step treatment of this slowly varying force). Default 1. */
int acs_engine_set_correction_stride(acs_engine* e, int32_t stride);
/* Mean duration (ms) of the correction launches in the last acs_engine_run_timed call. */
float acs_engine_last_correction_ms(acs_engine* e);
/* Nose-Hoover state per replica, (xi, eta) pairs in caller units (host array of 2 n_replicas): set = 0
 * reads it into xi_eta, set = 1 writes it from xi_eta (before a run, e.g. from the integrator object).
 * Synchronous. */
int acs_engine_nh_state(acs_engine* e, double* xi_eta, int32_t set);
/* Thermostat (bath) energy Q xi^2 / 2 + N_f kT eta at each record (Nose-Hoover; 0 otherwise): record i of
 * replica r at out_dev[i * n_replicas + r], device array. */
int acs_engine_bath_records(acs_engine* e, double* out_dev, int32_t count, void* stream);
int acs_engine_destroy(acs_engine* e);

#ifdef __cplusplus
}
#endif
#endif /* ACCUSIM_B200_ENGINE_H */
