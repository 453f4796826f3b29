/*
 * pyrocmc.h -- C ABI of the B200 (sm_100a) Monte Carlo engine for classical
 * Heisenberg spins on the pyrochlore lattice (libpyrocmc.so).
 *
 * This is the boundary the reference's C++ interfaces sit on: the C++ shims in
 * pyro_cmc_b200/host/ (CMC::MC_runner, ssf_manager, energy_manager) and the
 * Python bindings (pyro_cmc_b200/_lib.py) call only these functions. Every
 * function returns 0 (PC_OK) on success or a PC_ERR_* code; the message of the
 * last failure on the calling thread is returned by pc_last_error().
 *
 * Plain pointers and sizes only. "host" arrays are ordinary CPU memory;
 * "device" pointers are CUDA global memory on the system's device.
 *
 * Conventions (fixed by this library; the reference leaves them to lattice_lib):
 *   site index   i = sl * Nc + cell, sl = 4*f + p (16 sublattices, pyro_sl = p),
 *                cell = cx + L*(cy + L*cz), Nc = L^3, N = 16*Nc
 *                (sublattice-major like src/MC.cpp:32);
 *   position     x_i = 8*(cx,cy,cz) + R_fcc[f] + link[p]
 *                (include/pyrochlore_geometry.hpp:12-32);
 *   k points     K in [0,L)^3, q = 2*pi*K/(8L), flat k = (K0*L + K1)*L + K2;
 *   SSF          S^{ab}(q) = conj(B^a(q)) B^b(q), B^a(q) = sum_i exp(-i q.x_i) S^a_i
 *                (equal to ssf_manager's phase-contracted sum,
 *                include/ssf_manager.hpp:260-293, with a forward-signed,
 *                unnormalised DFT).
 *   RNG          Philox4x32-10, key = seed, counter = (site, sweep lo32,
 *                draw | sweep hi32 << 8, replica); draw 0 = Metropolis,
 *                1 = lifted Metropolis, 2+k = overrelaxation pass k,
 *                250 = random initial state, 251 = replica exchange. With
 *                u = top 24 bits / 2^24 of a word: Gaussian pair radius
 *                sqrt(-2 ln(u + 2^-24)), angles 2 pi (u - 1/2); Metropolis
 *                acceptance uniform = low bytes of words 0..2 / 2^24.
 */
#ifndef PYROCMC_H
#define PYROCMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PC_OK 0
#define PC_ERR_INVALID 1     /* bad argument (reference: std::invalid_argument / logic_error) */
#define PC_ERR_CUDA 2        /* CUDA runtime failure */
#define PC_ERR_STATE 3       /* call out of order (e.g. sweep before setup_lattice) */
#define PC_ERR_UNSUPPORTED 4 /* configuration this build does not handle */
#define PC_ERR_TIMEOUT 5     /* a bounded device-side wait gave up */

typedef struct pc_system pc_system;

/* Message of the last failure on this thread ("" if none). */
const char* pc_last_error(void);
/* Library ABI version (major*100 + minor). */
int pc_version(void);

/* ---------------------------------------------------------------- lifetime */

/* Creates n_replicas independent lattices of L[r]^3 cubic cells each (uneven L
 * allowed) on the current CUDA device. One replica is the reference's single
 * Lattice; several are the batched replicas that replace temper's MPI ranks.
 * Replaces MC_runner(Lattice&, size_t seed) (include/MC.hpp:107-112); the seed
 * is the Philox key, used as given (no seed-table lookup). */
int pc_create(int n_replicas, const int32_t* L, uint64_t seed, pc_system** out);
int pc_destroy(pc_system* sys);
/* Makes the system launch on an existing CUDA stream (cudaStream_t) instead of
 * its own, e.g. the caller's framework stream; the caller keeps ownership. */
int pc_set_stream(pc_system* sys, void* stream);

/* Replaces the Philox key (MC_runner is constructed with its seed after the
 * Lattice exists, include/MC.hpp:107). */
int pc_set_seed(pc_system* sys, uint64_t seed);

/* MC_runner::define_coupling (include/MC.hpp:121-124, src/MC.cpp:56-66).
 * rel_vecs: displacement vectors for pyro_sl 0..3 concatenated, n_rel[p] of
 * them for sublattice p, 3 int64 each. J: 3x3 row-major, applied by the source
 * (lower pyro_sl) endpoint; the target endpoint applies J^T.
 * Duplicate names fail with PC_ERR_INVALID ("Coupling names must be unique"). */
int pc_define_coupling(pc_system* sys, const char* name, const int64_t* rel_vecs, const int32_t* n_rel,
                       const double* J);
/* Replaces the matrix of coupling `spec` (definition order) after setup,
 * rebuilding the bond tables (and colour classes, which follow the nonzero
 * bonds). Used by the differentiable path to move J. */
int pc_set_coupling_matrix(pc_system* sys, int spec, const double* J);
/* The same for n couplings at once: specs[k] gets J[9k .. 9k + 8], and the
 * tables are rebuilt once; nothing is rebuilt when every matrix already
 * holds those values. PC_ERR_INVALID (nothing changed) for an index out of
 * range. */
int pc_set_coupling_matrices(pc_system* sys, int n, const int32_t* specs, const double* J);
/* MC_runner::set_global_field / get_global_field (include/MC.hpp:126-127). */
int pc_set_global_field(pc_system* sys, const double* B3);
int pc_get_global_field(pc_system* sys, double* B3);
/* MC_parameters::T_ref (include/MC.hpp:79-82): proposal width sqrt(T/T_ref). */
int pc_set_T_ref(pc_system* sys, double T_ref);
/* Overrelaxation form: 0 = random-angle rotation about the local field
 * (overrelax_all, src/MC.cpp:145-153; default), 1 = reflection
 * (mirror_about_vector, src/MC.cpp:98-100). */
int pc_set_overrelax_mode(pc_system* sys, int mode);
/* Colour classes of the sweep. 0 (default): one class per sublattice, in
 * sublattice order -- the sweep then visits sites in exactly the reference's
 * sequential storage order (spins[sl*Nc + cell], src/MC.cpp:157), so the Markov
 * chain is the reference's. 1: fewest classes (sublattices joined by no
 * nonzero bond share a class: 4 pyro_sl classes when J3 = 0); a different,
 * equally valid visiting order with fewer launches. Call before setup. */
int pc_set_colouring(pc_system* sys, int mode);
/* Sweep schedule. 0 (default): the reference's order -- a Metropolis pass
 * over all colour classes, then n_overrelax overrelaxation passes
 * (src/MC.cpp:155-163). 1 (fused): each colour pass applies the Metropolis
 * move and then the first overrelaxation move to every site of the class,
 * both with the site's local field, which no move of the pass changes; the
 * remaining n_overrelax - 1 passes follow as in schedule 0. Both moves keep the
 * Boltzmann distribution invariant, so the fused sweep samples the same
 * ensemble with one local-field evaluation per site instead of two. The
 * Philox draws per site are those of schedule 0. */
int pc_set_sweep_schedule(pc_system* sys, int schedule);
/* The single-site move of a sweep. 0 (default): local_Metropolis
 * (src/MC.cpp:111-130), sweep_local_Metropolis. 1: lifted Metropolis, u-form
 * (local_lifted_Metropolis, src/MC.cpp:249-281; sweep_lifted_Metropolis
 * :284-291, the move of `anneal --lifted`). 2: lifted Metropolis, rotation
 * form (local_lifted_Metropolis_rot, src/MC.cpp:194-244;
 * sweep_lifted_Metropolis_rot :293-302). The per-spin lifting direction
 * (include/MC.hpp:57) is the sign of the spin's fourth float4 component
 * (>= 0: +1); lifted passes and overrelaxation passes keep it, while
 * pc_set_spins and a Metropolis (non-lifted) pass reset it to +1. Lifted sweeps visit the classes in
 * the reference's order (a lifted pass, then the overrelaxation passes), for
 * either sweep schedule. */
int pc_set_update(pc_system* sys, int mode);
/* Kernel path: 0 (default) uses the structured pyrochlore kernels whenever the
 * couplings fit the fixed J1/J2/J3a/J3b neighbour structure, 1 forces the
 * generic bond-table kernels. Reports the path in use via pc_kernel_path. */
int pc_set_kernel_path(pc_system* sys, int force_generic);
int pc_kernel_path(pc_system* sys, int* structured);
/* MC_runner::setup_lattice (src/MC.cpp:15-52): builds the per-sublattice bond
 * shells, the colour classes and uploads them. Must follow all couplings. */
int pc_setup_lattice(pc_system* sys);

/* Pyrochlore displacement tables, derived from the geometry (the vectors d
 * with |d|^2 = 8, 24, 32 from a site of pyro_sl p to another site):
 * kind 1 = J1 (nn1_dist, include/pyrochlore_geometry.hpp:110-115),
 * 2 = J2 (nn2_dist, :117-134), 3 = J3a (nn3a_dist, :137-142; the midpoint is a
 * site), 4 = J3b (nn3b_dist, :144-149), 10 + nu = the J1 vectors from p that
 * land on pyro_sl nu (nn1_pair_MN, :151-190). Writes *n vectors (3 int64 each)
 * into out (room for max_n). */
int pc_pyrochlore_displacements(int kind, int pyro_sl, int64_t* out, int max_n, int* n);

/* ------------------------------------------------------------ inspection */

int pc_num_replicas(pc_system* sys, int* n);
int pc_num_spins(pc_system* sys, int replica, int64_t* n);
/* Colour classes used by the sweep: colour_of_sl[16]. */
int pc_colours(pc_system* sys, int* n_colours, int32_t* colour_of_sl);
/* Neighbour site indices of every site of a replica for coupling `spec`
 * (definition order), in that spec's displacement order: out[N][max_nb], -1
 * padded. The bit-exact geometry check against the reference tables. */
int pc_neighbour_table(pc_system* sys, int replica, int spec, int max_nb, int32_t* out);
/* ipos of each site (wrapped into [0, 8L)) and its sublattice. */
int pc_site_positions(pc_system* sys, int replica, int64_t* pos, int32_t* sl);
/* Number of kernels this system has launched so far (graph replays count
 * their kernel nodes). */
int pc_launch_count(pc_system* sys, uint64_t* n);

/* ----------------------------------------------------------------- spins */

/* Host <-> device spin state, N x 3 doubles (the Lattice mirror sync). */
int pc_set_spins(pc_system* sys, int replica, const double* S);
int pc_get_spins(pc_system* sys, int replica, double* S);
/* Same, in the device layout: N x 4 floats (x, y, z, unused). */
int pc_set_spins_f4(pc_system* sys, int replica, const float* S4);
int pc_get_spins_f4(pc_system* sys, int replica, float* S4);
/* Uniform on S^2 for every replica, drawn on the device (Philox draw 250). */
int pc_random_spins(pc_system* sys, uint64_t seed);
/* Device address of a replica's spin array (float4[N]); valid until destroy. */
int pc_spins_device(pc_system* sys, int replica, void** dev_ptr);
/* The per-replica sweep counter (Philox counter); settable for exact resume. */
int pc_get_sweep_counter(pc_system* sys, int replica, uint64_t* sweep);
int pc_set_sweep_counter(pc_system* sys, int replica, uint64_t sweep);

/* -------------------------------------------------------------------- MC */

/* MC_runner::sweep_local_Metropolis(T, n_overrelax) (src/MC.cpp:155-163) for
 * every replica at once, n_sweeps times: one Metropolis pass (Gaussian kick
 * of width sqrt(T/T_ref), renormalised, src/MC.cpp:111-130) then n_overrelax
 * overrelaxation passes, each over the colour classes in order.
 * T[r] per replica (host array). accepted[r] (host, may be NULL) receives the
 * accepted Metropolis moves summed over the n_sweeps sweeps. */
int pc_sweep(pc_system* sys, const double* T, int n_sweeps, int n_overrelax, uint64_t* accepted);
/* overrelax_all (src/MC.cpp:145-153) alone on every replica: one
 * overrelaxation pass over the colour classes with Philox angles (draw 2 at
 * the current sweep counter), then the counter advances by one. */
int pc_overrelax_all(pc_system* sys);
/* overrelax_all (src/MC.cpp:145-153) alone, with deterministic angles:
 * theta (host, N doubles for `replica`) or NULL for reflection. For parity
 * tests of one overrelaxation pass. */
int pc_overrelax_theta(pc_system* sys, int replica, const double* theta);
/* total_energy_per_unit_cell (src/MC.cpp:305-312) of every replica (host
 * e_per_cell[R]) and the magnetisation sum_i S_i (host mag[R][3], may be NULL).
 * FP64 accumulation. */
int pc_energy(pc_system* sys, double* e_per_cell, double* mag);
/* MC_runner::local_field (src/MC.cpp:87-96) of every site of a replica,
 * without the global field: host h[N][3]. */
int pc_local_field(pc_system* sys, int replica, double* h);

/* ------------------------------------------------------------------- SSF */

/* ssf_manager constructor (include/ssf_manager.hpp:161-201): the correlator
 * labels ("xx", "xy", ...; two of x/y/z each) and n_slots accumulator slots
 * (temperatures), each for replicas of size L_of_slot[slot]. Bad labels fail
 * with PC_ERR_INVALID and the reference's message. Clears all slots. */
int pc_ssf_configure(pc_system* sys, const char* const* names, int n_corr, int n_slots, const int32_t* L_of_slot);
/* Sublattice-resolved accumulators (resolved != 0): the correlator of
 * ssf_manager::sample before its phase contraction, C^{ab}_{mu nu}(k) =
 * conj(A^a_mu(k)) A^b_nu(k) with A^a_mu the DFT over cells of S^a on sublattice
 * mu (include/ssf_manager.hpp:260-293, correlate()), accumulated as sums and
 * (Re)^2, (Im)^2 sums in the layout [n_corr][n_k][16][16][2] per slot that
 * src/temper.cpp:121-159 writes to /ssf. 256x the memory of the contracted
 * form. Call before pc_ssf_configure (it invalidates a configured SSF); the
 * reads (pc_ssf_read, pc_ssf_current) then return the resolved layout.
 * Needs every L to factor into two parts <= 8 (L <= 64). */
int pc_ssf_set_resolved(pc_system* sys, int resolved);
/* Seed merge (scripts/acc_runs.py:228-370, merge_group) of K slots that hold
 * the same temperature for K seeds with the same sample count n, computed on
 * the device: static_corr = sum of the slots' S(q) sums, static_corr_2 = sum
 * of their squares, var_inter = static_corr_2/(K n^2) - (static_corr/(K n))^2,
 * var_intra = sum of the slots' square sums / n - static_corr_2 / n^2, each
 * [n_corr][n_k][2]; and per seed the spiral-plane invariants of
 * plane_invariants (:103-167) w, chi_frac and tr, each [K][n_k] (need the
 * correlators xx, yy, zz, xy, xz, yz). Every output may be null. */
int pc_ssf_merge(pc_system* sys, const int32_t* slots, int K, double* static_corr, double* static_corr_2,
                 double* var_inter, double* var_intra, double* w, double* chi_frac, double* tr);
/* ssf_manager::sample (include/ssf_manager.hpp:260-293) for every replica r
 * with slot_of_replica[r] >= 0 (host array): accumulates S(q) and
 * (Re S)^2, (Im S)^2 into that slot in FP64 and counts the sample. */
int pc_ssf_sample(pc_system* sys, const int32_t* slot_of_replica);
/* Copies a slot out: sum and sq as [n_corr][n_k][2] doubles, n_samples. */
int pc_ssf_read(pc_system* sys, int slot, double* sum, double* sq, uint64_t* n_samples);
int pc_ssf_clear(pc_system* sys, int slot);
/* S(q) of the current configuration of one replica, no accumulation:
 * out[n_corr][n_k][2] (host). */
int pc_ssf_current(pc_system* sys, int replica, double* out);

/* save_ft_spin_state (src/MC.cpp:320-368): the raw per-sublattice DFT over
 * cells of each spin component of one replica, WITHOUT the sublattice phase
 * exp(-i q.r_mu) (which the reference also leaves to post-processing):
 * out[3][16][n_k][2] (host; components x, y, z; sublattice sl = 4f + p;
 * k flat as above; re, im), A^a_sl(K) = sum_cells exp(-2 pi i K.n / L) S^a.
 * Computed on the device in FP32 (the transforms of the resolved S(q)),
 * returned in FP64. Needs L to factor into two parts <= 8 (L <= 64). */
int pc_spin_ft(pc_system* sys, int replica, double* out);

/* -------------------------------------------------------- tempering / energy */

/* Sets up batched parallel tempering over all replicas (replaces the MPI
 * ranks of src/temper.cpp). Replicas with equal L form a ladder; T[r] is the
 * initial temperature of replica r, and the ladder's slots are its
 * temperatures sorted descending (slot order = temper's rank order). Energy
 * accumulators (energy_manager, include/energy_manager.hpp:19-48) are kept per
 * slot. Exchange attempts are decided on the device. */
int pc_pt_configure(pc_system* sys, const double* T);
/* n_rounds rounds of: n_sweep sweeps at each replica's current temperature;
 * an SSF sample into the replica's slot whenever the sweep count reaches a
 * multiple of ssf_every (0 = never; needs pc_ssf_configure with one slot per
 * replica); one energy sample per slot; a checkerboard exchange attempt
 * between adjacent temperatures of every ladder (pairs (0,1),(2,3).. on even
 * rounds, (1,2),.. on odd, src/temper.cpp:437-473). The schedule is captured
 * as a CUDA graph and replayed. */
int pc_pt_run(pc_system* sys, int n_rounds, int n_sweep, int ssf_every);
/* Tempering rounds in one persistent cooperative launch (off by default): with
 * 1, pc_pt_run runs all its rounds -- every colour pass of every replica, the
 * energies and the exchanges -- in one kernel launch with grid barriers
 * between the phases (with S(q) samples: one launch per stretch of sweeps
 * between samples). Same site updates, draws and exchange rule as the
 * per-pass graph: the same chain, up to the rounding of the energy sums (one
 * thread per site here, one per cubic cell there), which the exchange
 * decisions see. PC_ERR_UNSUPPORTED for systems it does not cover
 * (non-pyrochlore couplings, lifted moves, reflection overrelaxation, the
 * staged row tiles, block sizes outside 32..256). No counterpart in the
 * reference (an execution strategy of src/temper.cpp:418-474). */
int pc_set_pt_persistent(pc_system* sys, int on);
int pc_get_pt_persistent(pc_system* sys, int* on);
/* Zeroes the energy accumulators and exchange statistics (after burn-in);
 * the replica-to-slot assignment and the spins are kept. */
int pc_pt_reset_stats(pc_system* sys);
/* Per-slot energy accumulators (sum e, sum e^2, count) and temperatures. */
int pc_pt_read_energy(pc_system* sys, double* T, double* E, double* E2, uint64_t* n);
/* Per-slot exchange statistics: attempts/accepts of the pair (slot, slot+1). */
int pc_pt_read_exchange(pc_system* sys, uint64_t* attempts, uint64_t* accepts);
/* Current slot of every replica. */
int pc_pt_slots(pc_system* sys, int32_t* slot_of_replica);

/* ------------------------------------------------------- differentiation */

/* Energy and its gradient for every replica (the autograd path). With upstream
 * scalar g[r] for e_per_cell[r]:
 *   grad_S[r][i] = g[r]/Nc * (h_i - B)            (device, float4[N_total], may be NULL)
 *   grad_J[r][spec][9] = g[r]/Nc * dE/dJ_spec      (host, may be NULL)
 *   grad_B[r][3] = -g[r]/Nc * sum_i S_i            (host, may be NULL)
 * and e_per_cell[r] (host). dE/dJ_spec[a][b] = sum over the spec's bonds of
 * S_src[a] S_tgt[b]. With grad_J NULL the coupling products are not formed at
 * all (the spin gradient alone costs about one energy evaluation). */
int pc_energy_grad(pc_system* sys, const double* g, double* e_per_cell, void* grad_S_dev, double* grad_J,
                   double* grad_B);
/* Device-output forms for callers that keep the results on the GPU (the
 * autograd path): the work is queued on the system's stream (pc_set_stream)
 * and the calls return without waiting for it; a device error flag raised by
 * these kernels is reported by the next call that waits.
 * pc_energy_device: e_dev[r] = e_per_cell[r] (R doubles, device).
 * pc_energy_grad_device: upstream g_dev[r] (R doubles, device; NULL: 1 for
 * every replica); grad_S as pc_energy_grad (may be NULL); sums_dev (may be
 * NULL) receives per replica a row of 4 + 9 * n_spec doubles: [sum over the
 * cells of the owned bond energies - S.B (= e_per_cell * Nc), sum_i S_i (3),
 * and with couplings != 0 the coupling products dE/dJ_spec (9 per spec, as
 * pc_energy_grad's grad_J before the factor g/Nc)]; without couplings the
 * products are not formed and those columns are left untouched. */
int pc_energy_device(pc_system* sys, double* e_dev);
/* pc_energy_device plus, per replica, out_dev[r][9] = [the bare sums of
 * S_i.S_j over the bonds of each of the six coupling groups (J1 towards
 * pyrochlore sublattices in three groups, J2, J3a, J3b), sum_i S_i (3)] (device,
 * queued without waiting): dE/dj of each group's isotropic coupling j I times
 * Nc, from the energy pass itself. PC_ERR_UNSUPPORTED unless every group
 * matrix is j I, j != 0, the same on all sublattices. */
int pc_energy_groups_device(pc_system* sys, double* e_dev, double* out_dev);
int pc_energy_grad_device(pc_system* sys, const double* g_dev, void* grad_S_dev, double* sums_dev, int couplings);
/* pc_energy_grad evaluated on an arbitrary field instead of the system's
 * spins: field_dev (device, float4[N_total], 16-byte aligned, any length per
 * site) stands for S in every formula above, with the system's couplings and
 * field. With g[r] = Nc the outputs are h_i(field) - B and the bond sums
 * sum field_src[a] field_tgt[b]; the differentiable gradient quench uses it
 * for the local field of an upstream gradient (the energy's Hessian is the
 * coupling matrix) and, through (P(S + v) - P(S) - P(v)), for the mixed bond
 * sums of its coupling gradient. No counterpart in the reference (the
 * backward of MC_runner::local_field, src/MC.cpp:87-96). grad_S_dev must not
 * alias field_dev. */
int pc_energy_grad_field(pc_system* sys, const void* field_dev, const double* g, double* e_per_cell,
                         void* grad_S_dev, double* grad_J, double* grad_B);
/* S(q) for every replica into a device buffer out_dev[R][n_corr][n_k][2]
 * (float64), no accumulation. Uses the correlators of pc_ssf_configure. */
int pc_ssf_forward(pc_system* sys, void* out_dev);
/* Backward of pc_ssf_forward: given dLoss/dS (device, same layout as
 * out_dev: d/dRe, d/dIm), writes dLoss/dS_i into grad_S_dev (float4[N_total],
 * device). Recomputes the forward transform instead of storing it (see
 * pc_ssf_backward_kept). */
int pc_ssf_backward(pc_system* sys, const void* grad_out_dev, void* grad_S_dev);
/* The same pair for callers that keep the results on the GPU (the autograd
 * path): both are queued on the system's stream (pc_set_stream) and return
 * without waiting. pc_ssf_forward_keep also keeps the forward amplitudes and
 * hands out a token (nonzero) for them; pc_ssf_backward_kept with that token
 * uses them instead of recomputing the forward transform, provided the
 * system's spins are again those of that forward (the caller's contract, as
 * with a tensor saved for backward) and no forward or backward ran in
 * between (else the token is stale and the transform is recomputed). */
int pc_ssf_forward_keep(pc_system* sys, void* out_dev, uint64_t* token);
int pc_ssf_backward_kept(pc_system* sys, uint64_t token, const void* grad_out_dev, void* grad_S_dev);

/* ------------------------------------------------------ allocation-free */

/* No counterpart in the reference. Energy per cubic cell and magnetisation of
 * one pyrochlore lattice for callers that may not allocate device memory: a
 * program whose device memory belongs to a framework's caching allocator (an
 * allocation behind its back fragments the pool, or fails once the pool holds
 * the free memory), or a loop that cannot absorb the device-wide
 * synchronisation of cudaFree. Nothing is allocated: the reduction's partial
 * sums live in a 512 KiB array compiled into the library, shared by all calls
 * on a device and kept until the process exits.
 *   spins_dev  device, float4[16 L^3] in this library's site order, 16-byte
 *              aligned
 *   L          1..64 (larger L is rejected with PC_ERR_INVALID before any work)
 *   params     host, 7 doubles: J1, J2, J3, Delta, Bx, By, Bz (the coupling set
 *              of build_J1J2J3_h)
 *   out_dev    device, 4 doubles, 8-byte aligned: energy per cubic cell,
 *              sum_i S_i (x, y, z)
 *   stream     cudaStream_t to launch on (NULL: the default stream)
 * Misaligned pointers are rejected with PC_ERR_INVALID. Asynchronous on
 * `stream`. The first call in a CUDA context (the first on a device, and the
 * first after that device's context is re-created, e.g. by cudaDeviceReset)
 * looks up the scratch array's address; make it before any stream capture.
 * Calls that overlap on the GPU (e.g. on two streams) race on the shared
 * array. */
int pc_energy_noalloc(const void* spins_dev, int L, const double* params, void* out_dev, void* stream);

/* ------------------------------------------------------------------ tuning */

/* Times the sweep over the candidate tile shapes (threads per CTA x CTAs per
 * SM) and neighbour-load variants on this system, and the cluster-resident
 * sweep where it applies, then launch overlap off and on for the chosen tile,
 * and keeps the fastest (spin state and sweep counter are saved and
 * restored). */
int pc_autotune(pc_system* sys);
/* How the structured kernels issue the 30 neighbour loads of a site:
 * 0 group by group (fewest registers), 1 all at once, 2 in two batches, 3 staged:
 * a CTA copies the 24 neighbour-row blocks of its tile of x-rows into shared
 * memory with bulk asynchronous copies (L <= threads <= 256; else variant 0). */
int pc_set_load_variant(pc_system* sys, int variant);
int pc_get_load_variant(pc_system* sys, int* variant);
/* Current tile shape (threads per CTA, CTAs per SM). CTAs per SM = 0 launches
 * one CTA per tile instead of a grid of SMs x CTAs striding over the tiles. */
int pc_get_tile(pc_system* sys, int* threads, int* ctas_per_sm);
int pc_set_tile(pc_system* sys, int threads, int ctas_per_sm);

/* --------------------------------------------------------------- bench API */

/* One end-to-end step through host buffers: copies S4_in (host, N x 4 floats,
 * pinned for full speed) to replica 0, runs n_sweep sweeps at temperature T
 * with an SSF sample into ssf_slot after every ssf_every sweeps (ssf_slot < 0
 * or ssf_every = 0: none), takes one energy sample, and copies the spins back
 * to S4_out and the energy per cell to *e_out. */
int pc_step_host(pc_system* sys, const float* S4_in, float* S4_out, double T, int n_sweep, int ssf_every,
                 int ssf_slot, double* e_out, uint64_t* accepted);
/* The same step with host spins as N x 3 floats (x, y, z per site, the three
 * components of the reference's HeisenbergSpin::S, include/MC.hpp:55): 12
 * bytes a spin cross the bus instead of 16. The spins are unpacked and packed
 * on the device; the lifting directions of lifted Metropolis (the fourth
 * float4 component) stay on the device. Same chain and results as
 * pc_step_host given the same spins. */
int pc_step_host3(pc_system* sys, const float* S3_in, float* S3_out, double T, int n_sweep, int ssf_every,
                  int ssf_slot, double* e_out, uint64_t* accepted);
/* CUDA events around the last pc_sweep call's kernels: average duration in
 * milliseconds of the Metropolis and overrelaxation colour-pass kernels. */
int pc_last_kernel_times(pc_system* sys, double* metropolis_ms, double* overrelax_ms);
/* Luttinger-Tisza bound (src/luttinger_tisza.cpp, the ltgs program): for
 * every k = 2 pi K / (8L) of the L^3 grid the smallest eigenvalue of the
 * 48 x 48 Hermitian M(k) = sum over directed bonds J_bond exp(i k.d)
 * (build_bonds :31-81: J1 XXZ, J2, J3a, J3b; zero couplings skipped;
 * :153-178), on the GPU in FP64. Outputs (each may be null):
 * lambda_map[L^3] (flat C order over K, the reference's eigenvalue_map),
 * *e_per_spin = lambda_min / 2 (:181, the reference's E_min), k_star[3] = the
 * first K in flat order attaining the minimum, eigvec[48][2] = a unit
 * eigenvector there (rows spin-x,y,z of sublattice 0, 1, ...). Uses the
 * current device; needs no pc_system. */
int pc_lt_minimum(int L, double J1, double J2, double J3, double Delta, double* lambda_map, double* e_per_spin,
                  int64_t* k_star, double* eigvec);
/* Bound of the first wait of the staged colour pass (load variant 3) on its
 * bulk copies, in polls of a hardware-timed try_wait (default and maximum
 * 2^22; < 0 restores the default), and of every grid-barrier wait of the
 * persistent tempering kernel, in polls of ~64 ns (default and maximum 2^24).
 * For tests of the timeout paths: with 0 every staged pass gives up at once,
 * sets the device error flag, waits for its copies at the full bound (none is
 * left in flight), skips its updates, and the call returns PC_ERR_TIMEOUT; a
 * persistent tempering launch gives up at its first barrier and every block
 * leaves (the round is left unfinished), PC_ERR_TIMEOUT. The system stays
 * usable. No counterpart in the reference (it has no device waits). */
int pc_set_wait_limit(pc_system* sys, int polls);
/* Enables per-kernel CUDA-event timing (off by default). */
int pc_set_kernel_timing(pc_system* sys, int on);
/* Launch overlap of consecutive colour passes (off by default; pc_autotune
 * turns it on where it is faster): with 1 each pass is launched with
 * programmatic dependent launch and waits in-kernel for the previous kernel's
 * completion before reading spins, so its launch overlaps the previous pass's
 * last CTAs. Measured on B200: 3-4 % faster sweeps for L = 8..32, nothing at
 * L = 64. Results are identical either way. No counterpart in the reference
 * (a launch setting). */
int pc_set_launch_overlap(pc_system* sys, int on);
/* Cluster-resident sweeps (off by default; pc_autotune turns them on where
 * they are faster): for replicas of one size L <= 16, one thread-block cluster
 * of L CTAs per replica holds the lattice in distributed shared memory (one z
 * plane of all 16 sublattices per CTA) and runs every colour pass of a
 * pc_sweep call in one launch, with a cluster barrier between passes. Same
 * passes, draws and arithmetic as the per-pass kernels: the same chain.
 * PC_ERR_UNSUPPORTED when the system does not qualify (other sizes, lifted
 * moves, non-pyrochlore couplings, no cluster of that size fits). No
 * counterpart in the reference (an execution strategy of
 * MC_runner::sweep_local_Metropolis, src/MC.cpp:155-163). */
int pc_set_cluster_sweeps(pc_system* sys, int on);
int pc_get_cluster_sweeps(pc_system* sys, int* on);

#ifdef __cplusplus
}
#endif
#endif /* PYROCMC_H */
