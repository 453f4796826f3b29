// kernels.h -- launch interface between the host system (system.cu) and the
// kernels (sweep.cu, ssf.cu, pt.cu). Plain structs, no torch types.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "pyro_struct.cuh"

namespace pc {

// kFused*: the Metropolis move and then one overrelaxation move of the same
// site in one pass, both with the site's local field (which no move of this
// pass changes).
enum PassMode {
    kMetropolis = 0,
    kOverrelaxRotate = 1,
    kOverrelaxReflect = 2,
    kOverrelaxTheta = 3,
    kFusedRotate = 4,
    kFusedReflect = 5,
    kLifted = 6,     // lifted Metropolis, u-form (src/MC.cpp:249-281)
    kLiftedRot = 7   // lifted Metropolis, rotation form (src/MC.cpp:194-244)
};

// Internal load variants: variant 0 with the isotropic group-matrix path and
// no per-group activity test, used by the host when every group matrix is
// j I with j != 0 (kVarIso), or when that holds for every group but the J2
// group, whose matrix is 0 everywhere (kVarIsoNoJ2: J2 = 0).
constexpr int kVarIso = 5, kVarIsoNoJ2 = 6;
// Or'ed into a load variant (0, kVarIso, kVarIsoNoJ2): spins, own spin and
// temperature are read with ordinary weak loads instead of the read-only path,
// for a kernel that writes them in an earlier phase of the same launch (the
// persistent tempering kernel, whose grid barrier orders the phases).
constexpr int kVarCoherent = 0x100;
// Or'ed into kVarIso by the per-pass fused rotation kernel: neighbour
// addresses from per-sublattice bases (load_nb's UB form).
constexpr int kVarUniformBase = 0x200;
// The per-replica constants of a Metropolis proposal at temperature T: the
// kick width sqrt(T / T_ref) and 1 / T, rounded as the moves use them. Formed
// once per replica whenever the temperatures change, not per site.
__host__ __device__ inline float2 proposal_consts(double T, float inv_T_ref) {
    return make_float2(sqrtf(float(T) * inv_T_ref), float(1.0 / T));
}

struct PassArgs {
    float4* spins;
    const ReplicaDev* reps;
    const double* T_rep;         // per-replica temperature (device)
    const float2* Tq;            // per replica (sqrt(T / T_ref), 1 / T): proposal_consts of T_rep (device)
    const uint64_t* sweep_base;  // device sweep counter
    uint64_t sweep_offset;       // added to *sweep_base
    uint64_t seed;
    PhiloxKeys rkeys;  // the seed's Philox round keys (philox_round_keys)
    float inv_T_ref;
    float B[3];
    const SlTable* tables;  // 16 sublattice tables (device)
    int n_tab;              // sublattices of this colour
    int tab_sl[4];
    const Tile* tiles;
    int n_tiles;
    unsigned long long* acc;  // per-replica accepted Metropolis moves (device)
    int or_pass;              // overrelaxation pass index (draw 2 + or_pass)
    const double* theta;      // kOverrelaxTheta: per-site angle of replica theta_replica (device)
    int theta_replica;
    int structured;    // 1: couplings fit the pyrochlore structure, use `mats`
    int load_variant;  // structured path: how neighbour loads are batched (0, 1, 2), 3 = staged rows
    PyroMats mats;
    int staged_rl;  // load variant 3: largest tile (rows x L sites); sizes the shared row blocks
    int* err;       // device error flag (set by a kernel whose bounded wait ran out)
    int wait_polls; // load variant 3: polls of the first wait on the staged copies (kStagedMaxPolls)
};
// Bound of every wait of the staged pass on its bulk copies (polls of a
// hardware-timed try_wait).
constexpr int kStagedMaxPolls = 1 << 22;

// pdl: launch with programmatic dependent launch (the kernel waits for the
// previous kernel on the stream with griddepcontrol.wait before touching spins)
void launch_colour_pass(PassMode mode, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl = false);
// Load variant 3 (row tiles staged by bulk copies): sets the kernels' shared-memory limit.
void staged_prepare();
// The colour pass of load variant 3 (sweep_staged.cu) and of the lifted moves (sweep_lifted.cu).
void launch_staged(PassMode mode, const PassArgs& a, int threads, cudaStream_t st, bool pdl);
void launch_lifted_pass(PassMode mode, const PassArgs& a, int grid, int threads, cudaStream_t st, bool pdl);

// Cluster-resident sweeps (sweep_cluster.cu): one thread-block cluster per
// replica holds the whole lattice in distributed shared memory, one z plane of
// all 16 sublattices per CTA (cluster size L, L*L threads per CTA), and runs
// every colour pass of n_sweeps sweeps in one launch, a cluster barrier
// between passes. For replicas of one size L <= 16.
struct ClusterArgs {
    float4* spins;
    const ReplicaDev* reps;
    const double* T_rep;
    const uint64_t* sweep_base;  // device sweep counter (sweeps run at *sweep_base + 0 .. n_sweeps-1)
    uint64_t seed;
    float inv_T_ref;
    float B[3];
    unsigned long long* acc;  // per-replica accepted Metropolis moves
    PyroMats mats;
    int L;
    int n_sweeps;
    int n_or;       // overrelaxation moves per site per sweep
    int fused;      // 1: first round fused Metropolis + overrelaxation (n_or >= 1)
    int reflect;    // overrelaxation by reflection instead of a random-angle rotation
    int n_classes;  // colour classes in order, each up to 4 mutually unbonded sublattices
    int class_n[16];
    int class_sl[16][4];
};
// Shared memory per CTA of the cluster kernels for lattice size L.
size_t cluster_smem_bytes(int L);
// Prepares the kernels (cluster size and shared-memory attributes) and
// reports how many clusters of this size can be resident (0: not launchable).
int cluster_capacity(int L, int fused, int reflect);
void launch_cluster_sweeps(const ClusterArgs& a, int R, cudaStream_t st);

struct EnergyArgs {
    const float4* spins;
    const ReplicaDev* reps;
    const SlTable* tables;  // 16 tables
    const Tile* tiles;      // all sublattices of all replicas, replica-contiguous
    const int32_t* order;   // tiles in execution order, sublattice by sublattice
    int n_tiles;
    float B[3];
    double* partial;  // [n_tiles][4] by tile index: sum (0.5 S.h - S.B), sum S
    int structured;
    int iso;  // 1: every group matrix is j I with j != 0; 2: so but the J2 group, which is 0
    PyroMats mats;
};
void launch_energy_partials(const EnergyArgs& a, int threads, cudaStream_t st);
// Sums the tile partials of each replica in tile order: e[r] = sum/Nc, mag[r][3].
void launch_energy_finalize(const double* partial, const int32_t* tile_begin, const int32_t* tile_end,
                            const ReplicaDev* reps, int R, double* e, double* mag, cudaStream_t st);

// Energy with one thread per cubic cell (energy_cell.cu): tiles of up to
// kEnergyCellThreads consecutive cells of one replica, (replica, first cell,
// cells, 0); partial[tile][4] = sum of the owned bond energies - S.B, sum S.
constexpr int kEnergyCellThreads = 128;
struct EnergyCellArgs {
    const float4* spins;
    const ReplicaDev* reps;
    const int4* tiles;
    int n_tiles;
    float B[3];
    double* partial;
    int iso;  // as EnergyArgs::iso
    int uniform;  // iso != 0 and every group's j the same on all 16 sublattices: per-group bond sums
    PyroMats mats;
    double* group_partial;  // uniform only, or null: [n_tiles][kGroups] bare sums of S_i.S_j per group
};
void launch_energy_cells(const EnergyCellArgs& a, cudaStream_t st);

struct FieldArgs {
    const float4* spins;
    const ReplicaDev* reps;
    const SlTable* tables;
    const Tile* tiles;
    int n_tiles;
    float4* h_out;  // local field per site (global float4 layout), no global field
};
void launch_local_field(const FieldArgs& a, int threads, cudaStream_t st);

struct GradArgs {
    const float4* spins;
    const ReplicaDev* reps;
    const SlTable* tables;  // full tables (zero shells kept)
    const Tile* tiles;
    int n_tiles;
    int n_spec;
    float B[3];
    const double* g;   // per-replica upstream scalar (device)
    float4* grad_S;    // may be null
    double* partial;   // [n_tiles][4 + 9*n_spec]
};
void launch_energy_grad_partials(const GradArgs& a, int threads, cudaStream_t st);
void launch_grad_finalize(const double* partial, int width, const int32_t* tile_begin, const int32_t* tile_end,
                          int R, double* out /*[R][width]*/, cudaStream_t st);

// Structured energy gradient (grad.cu): work items of up to kGradK
// consecutive tiles of one (replica, sublattice), one site per tile and thread.
constexpr int kGradK = 2;
struct GradStructArgs {
    const float4* spins;
    const ReplicaDev* reps;
    const Tile* tiles;
    const int4* items;  // x = first tile, y = number of tiles (1..kGradK), z = partial-sum slot
    int n_items;
    int width;          // 4 (energy, sum S) or 4 + 9*n_spec (with dE/dJ per spec)
    float B[3];
    const double* g;    // per-replica upstream scalar (device)
    float4* grad_S;     // may be null
    double* partial;    // [n_items][width], by slot
    PyroMats mats;
    uint32_t spec_mask[16][kGroups][2];  // specs owning group g's side-k displacements
};
void launch_energy_grad_struct(const GradStructArgs& a, bool want_J, int threads, cudaStream_t st);

void launch_random_spins(float4* spins, const ReplicaDev* reps, const Tile* tiles, int n_tiles, uint64_t seed,
                         int threads, cudaStream_t st);
void launch_advance_counter(uint64_t* counter, uint64_t n, cudaStream_t st);

// ------------------------------------------------------------------ SSF
struct SsfGeom {
    int L;
    int P, Q;  // L = P*Q, two-level Cooley-Tukey split
    int n_rep;
    const int32_t* rep_index;  // replicas of this size (device)
    int resolved = 0;          // 1: sublattice-resolved correlators [n_corr][n_k][16][16][2]
};

// Raises the dynamic shared-memory limits of the SSF kernels (once, host side).
void ssf_prepare();
// Stage 1: per (replica, z-plane, z-group): xy DFT of the 4 sublattices of the
// group, times their xy sublattice phases, summed. G[rep][3][4][L][L][L] float2.
void launch_ssf_xy(const SsfGeom& g, const float4* spins, const ReplicaDev* reps, float2* G, cudaStream_t st);
// Stage 2 outputs.
struct SsfOut {
    int n_corr;
    int corr_a[9], corr_b[9];
    // accumulate mode: sum/sq [slot][n_corr][n_k][2] doubles ([slot][n_corr][n_k][16][16][2]
    // when resolved), slot per replica
    double* acc_sum;
    double* acc_sq;
    const int32_t* slot_of_rep;  // indexed by replica index
    int64_t slot_stride;         // doubles per slot (n_corr*n_k*2)
    // value mode: S(q) per replica into val[rep_pos][n_corr][n_k][2]
    double* val;
    // amplitude mode: B^a(K) per replica into amp[rep_pos][3][n_k] float2
    float2* amp;
};
void launch_ssf_z(const SsfGeom& g, const float2* G, const SsfOut& o, cudaStream_t st);
// The per-sublattice transforms alone (after launch_ssf_xy with resolved = 1):
// the z-DFT in place, leaving A[rep][3 * 16 (component, sublattice)][Kz][Ky][Kx]
// (float2), the raw DFT over cells of each component on each sublattice.
void launch_ssf_zdft_res(const SsfGeom& g, float2* A, cudaStream_t st);
// Whether line lengths P, Q have the fixed-radix (resolved-capable) kernels.
bool ssf_resolved_supported(int P, int Q);
// Backward: Y^c(K) from upstream dS (val layout) and amplitudes; then adjoint
// transform into grad_S (float4 per site, xyz components written).
void launch_ssf_adjoint(const SsfGeom& g, const SsfOut& o, const double* dval, const float2* amp, float2* H,
                        float4* grad_S, const ReplicaDev* reps, cudaStream_t st);

// ------------------------------------------------------------- tempering
struct PtArgs {
    int n_ladders;
    const int32_t* ladder_begin;  // slots of ladder l: [ladder_begin[l], ladder_begin[l+1])
    const double* T_slot;         // temperature of each slot
    int32_t* rep_of_slot;
    int32_t* slot_of_rep;
    double* T_rep;           // updated: T_rep[r] = T_slot[slot_of_rep[r]]
    float2* Tq;              // updated with T_rep: proposal_consts(T_rep[r], inv_T_ref)
    float inv_T_ref;
    const double* e_rep;     // energy per cell of each replica
    const ReplicaDev* reps;  // for Nc
    double* E_sum;           // per slot
    double* E2_sum;
    unsigned long long* n_e;
    unsigned long long* attempts;  // per lower slot
    unsigned long long* accepts;
    uint64_t* round;  // device round counter (parity + Philox counter)
    uint64_t seed;
    int n_slots;
};
void launch_pt_exchange(const PtArgs& a, cudaStream_t st);
// Tq[r] = proposal_consts(T[r], inv_T_ref) for r < R (sweep.cu).
void launch_refresh_tq(const double* T, float2* q, int R, float inv_T_ref, cudaStream_t st);

// Packed host spins (hostio.cu): (x, y, z) x n <-> the first three float4
// components; unpacking keeps each spin's fourth component.
void launch_spins_from_xyz(float4* spins, const float* xyz, int64_t n, cudaStream_t st);
void launch_spins_to_xyz(float* xyz, const float4* spins, int64_t n, cudaStream_t st);

// Tempering rounds of a batch of replicas in one persistent cooperative launch
// (pt_persistent.cu): per round, n_sweep sweeps (every colour pass of every
// replica; a grid barrier between passes), then, with `exchange`, the energy
// of every replica, its per-replica sum and the exchange round, each phase
// behind a grid barrier. The barrier's waits are bounded: when one runs out
// the kernel sets *err = kErrGridBarrier and every block leaves.
constexpr int kErrGridBarrier = 2;
// Grid barrier state: [0] top arrivals, [1] generation, then kBarrierGroups
// sub-counters, kBarrierStride words apart (one 128-byte line each).
constexpr int kBarrierGroups = 32, kBarrierStride = 32;
constexpr int kBarrierWords = kBarrierStride * (1 + kBarrierGroups);
struct PersistArgs {
    PassArgs pass;  // pass arguments (tiles, n_tiles, sweep_offset, or_pass unused)
    const Tile* colour_tiles[16];
    int n_colour_tiles[16];
    int n_colours;
    int fused;  // 1: one fused Metropolis + rotation pass per colour; 0: Metropolis passes, then rotation passes
    int n_rounds, n_sweep;
    int exchange;       // 1: energy + exchange after each round's sweeps
    uint64_t* sweep;    // device sweep counter: read at entry, advanced by n_rounds * n_sweep at exit
    // energy: one thread per cubic cell (cell_energy), tiles as EnergyCellArgs
    const int4* c_tiles;
    int n_c_tiles;
    int uniform;      // as EnergyCellArgs::uniform
    double* partial;  // [n_c_tiles][4]
    const int32_t* c_begin;  // replica r's cell tiles: [c_begin[r], c_end[r])
    const int32_t* c_end;
    double* e;    // per replica energy per cell
    double* mag;  // per replica sum of S
    int R;
    PtArgs pt;
    unsigned int* bar;  // [kBarrierWords], zero before the launch
    int max_polls;      // bound of each barrier wait (polls of ~64 ns)
};
// Blocks that fit on the device at once for this block size (0: unsupported).
int pt_persistent_capacity(int iso, int fused, int threads);
int launch_pt_persistent(const PersistArgs& a, int iso, int grid, int threads, cudaStream_t st);

// Seed merge of S(q) accumulators and spiral-plane invariants (merge.cu).
struct MergeArgs {
    const double* sum;   // [slot][n_corr][n_k][2]
    const double* sq;
    int64_t slot_stride;
    const int32_t* slots;  // K slot indices (device)
    int K, n_corr, n_k;
    double n;              // samples per seed
    int ix[6];             // correlator index of xx, yy, zz, xy, xz, yz, or -1
    double* out_corr;      // [n_corr][n_k][2]
    double* out_corr2;
    double* out_var_inter;
    double* out_var_intra;
    double* w;             // [K][n_k] (plane invariants; null: skipped)
    double* chi;
    double* tr;
    unsigned long long* max_bits;  // [K][2]: bits of max_k I2^{3/2}, max_k tr (non-negative doubles)
};

void launch_ssf_merge(const MergeArgs& a, cudaStream_t st);

}  // namespace pc
