// system.cu -- host side of libpyrocmc.so: the C ABI of include/pyrocmc.h.
//
// Owns the device state of a batch of replicas (spins, bond tables, colour
// tiles, SSF and tempering accumulators), builds the structured bond tables
// from reference-style coupling specs (MC_runner::setup_lattice,
// src/MC.cpp:15-52) and launches the kernels of sweep.cu / ssf.cu / pt.cu on
// the system's stream, replaying captured CUDA graphs for the sweep schedule.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pyrocmc.h"
#include "common.cuh"
#include "kernels.h"
#include "pyro_struct.cuh"

using pc::NbEntry;
using pc::ReplicaDev;
using pc::SlTable;
using pc::Tile;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define PC_CK(expr)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (expr);                                                                      \
        if (e_ != cudaSuccess) return fail(PC_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define PC_LAUNCH_CK()                                                                                \
    do {                                                                                              \
        cudaError_t e_ = cudaGetLastError();                                                          \
        if (e_ != cudaSuccess) return fail(PC_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    } while (0)

// Geometry of the 16-site cubic cell (include/pyrochlore_geometry.hpp:12-32).
const int64_t kLink[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
const int64_t kFcc[4][3] = {{0, 0, 0}, {0, 4, 4}, {4, 0, 4}, {4, 4, 0}};

int64_t pmod(int64_t a, int64_t m) {
    int64_t r = a % m;
    return r < 0 ? r + m : r;
}
std::array<int64_t, 3> r_sl(int sl) {
    const int f = sl / 4, p = sl % 4;
    return {kLink[p][0] + kFcc[f][0], kLink[p][1] + kFcc[f][1], kLink[p][2] + kFcc[f][2]};
}
// Sublattice of a position (any integer coordinates), -1 if no site.
int sl_at(const std::array<int64_t, 3>& x) {
    for (int sl = 0; sl < 16; ++sl) {
        const auto r = r_sl(sl);
        if (pmod(x[0] - r[0], 8) == 0 && pmod(x[1] - r[1], 8) == 0 && pmod(x[2] - r[2], 8) == 0) return sl;
    }
    return -1;
}

struct Coupling {
    std::string name;
    std::vector<std::array<int64_t, 3>> rel[4];
    double J[9];
    double Jt[9];
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    // on failure the buffer stays empty (p null, n 0): a later size check
    // allocates again instead of trusting a size that was never allocated
    cudaError_t alloc(size_t count) {
        release();
        if (count == 0) return cudaSuccess;
        const cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess)
            n = count;
        else
            p = nullptr;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

struct SsfGroup {
    int L, P, Q;
    std::vector<int> reps;
    DevBuf<int32_t> d_rep_index;  // all replicas of this size
    DevBuf<int32_t> d_sel_index;  // the replicas selected by the last sample call (capacity reps)
    int n_sel = 0;
    DevBuf<float2> d_G;           // stage-1 planes / adjoint scratch
    DevBuf<float2> d_amp;         // amplitudes B^a(K) for the backward
};

void split_PQ(int L, int* P, int* Q) {
    int best = 1;
    for (int p = 1; p * p <= L; ++p)
        if (L % p == 0) best = p;
    *P = best;
    *Q = L / best;
}

}  // namespace

namespace pc {
// lets the other translation units of the library report through pc_last_error()
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace pc

// Bound of each grid-barrier wait of the persistent tempering kernel, in
// polls of ~64 ns (about a second; a colour pass of the largest batches takes
// well under a millisecond).
constexpr int kBarrierMaxPolls = 1 << 24;

struct pc_system {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = true;

    int R = 0;
    std::vector<int> L;
    std::vector<int64_t> off;
    int64_t N_tot = 0;
    uint64_t seed = 0;
    double T_ref = 1.0;
    double B[3] = {0, 0, 0};
    int or_mode = 0;
    int colouring = 0;
    int schedule = 0;  // 0: Metropolis pass then overrelaxation passes; 1: fused
    std::vector<Coupling> specs;
    bool ready = false;

    SlTable tab_active[16];
    SlTable tab_full[16];
    bool structured = false;  // couplings fit the compile-time pyrochlore structure
    bool force_generic = false;
    pc::PyroMats mats;
    int n_colours = 0;
    int colour_of_sl[16];
    std::vector<std::vector<int>> colour_sls;

    int threads = 256;
    int ctas_per_sm = 4;
    int load_variant = 0;  // structured kernels: neighbour-load batching

    DevBuf<ReplicaDev> d_reps;
    DevBuf<float4> d_spins;
    DevBuf<double> d_T;
    DevBuf<float2> d_Tq;  // proposal_consts of d_T, refreshed before each batch of sweeps
    DevBuf<uint64_t> d_sweep;
    DevBuf<unsigned long long> d_acc;
    DevBuf<int> d_err;  // set by a kernel whose bounded wait ran out
    DevBuf<float> d_stage3;  // pc_step_host3: replica 0's spins as packed (x, y, z)
    int staged_rl = 0;  // load variant 3: largest row tile (R*L sites)
    int wait_polls = pc::kStagedMaxPolls;  // load variant 3: bound of the first wait (pc_set_wait_limit)
    DevBuf<SlTable> d_tab_active, d_tab_full;
    std::vector<DevBuf<Tile>> d_colour_tiles;
    std::vector<int> n_colour_tiles;
    DevBuf<Tile> d_all_tiles;
    DevBuf<int32_t> d_all_order;  // all tiles sublattice by sublattice (execution order of the energy)
    int n_all_tiles = 0;
    std::vector<int32_t> tile_begin, tile_end;
    DevBuf<int32_t> d_tile_begin, d_tile_end;
    DevBuf<double> d_partial;
    // energy with one thread per cubic cell (energy_cell.cu): tiles of cells
    // per replica, their ranges and FP64 partials
    DevBuf<int4> d_cell_tiles;
    int n_cell_tiles = 0;
    DevBuf<int32_t> d_cell_begin, d_cell_end;
    DevBuf<double> d_cell_partial;
    DevBuf<double> d_e, d_mag;
    DevBuf<double> d_theta;
    DevBuf<float4> d_field;
    DevBuf<double> d_grad_g, d_grad_out;  // energy-gradient upstream scalars and results
    DevBuf<double> d_grad_ones;           // g = 1 per replica (pc_energy_grad_device without g)
    DevBuf<double> d_group_partial, d_group_out;  // per-group bond sums (pc_energy_groups_device)
    // structured energy gradient: specs per (sublattice, group, bond side) and
    // work items of up to kGradK tiles of one (replica, sublattice)
    bool grad_struct = false;
    int iso_kind = 0;  // 1: every group matrix j I, j != 0; 2: so but a zero J2 group (isotropic variants)
    bool iso_uniform = false;  // iso_kind != 0 and each group's j the same on every sublattice
    uint32_t spec_mask[16][pc::kGroups][2] = {};
    DevBuf<int4> d_grad_items;
    int n_grad_items = 0;
    std::vector<int32_t> item_begin, item_end;
    DevBuf<int32_t> d_item_begin, d_item_end;
    DevBuf<double> d_grad_partial;

    uint64_t host_sweep = 0;
    uint64_t launches = 0;

    // sweep graph cache, keyed by n_overrelax
    std::map<std::pair<int, int>, std::pair<cudaGraphExec_t, int>> sweep_graphs;  // (n_or, sweeps) -> (graph, nodes)
    bool pdl = false;  // colour passes launched with programmatic dependent launch (measured: no gain)
    bool cluster_sweep = false;  // sweeps of small lattices in one cluster-resident launch (sweep_cluster.cu)
    std::map<std::array<int, 3>, int> cluster_cap;  // (L, fused, reflect) -> resident clusters (0: not launchable)
    int update = 0;   // 0 Metropolis, 1 lifted (u-form), 2 lifted (rotation form)

    // kernel timing
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    std::vector<int> ev_kind;  // 0 Metropolis, 1 overrelaxation
    size_t ev_used = 0;

    // SSF
    bool ssf_ready = false;
    int n_corr = 0;
    int corr_a[9], corr_b[9];
    int n_slots = 0;
    std::vector<int> L_of_slot;
    int64_t slot_stride = 0;
    bool ssf_resolved = false;  // sublattice-resolved accumulators [n_corr][n_k][16][16][2]
    DevBuf<double> d_ssf_sum, d_ssf_sq;
    std::vector<uint64_t> ssf_n;
    std::vector<SsfGroup> groups;
    DevBuf<int32_t> d_slot_of_rep;

    // tempering
    bool pt_ready = false;
    int n_ladders = 0;
    std::vector<int32_t> ladder_begin;
    std::vector<double> T_slot;
    DevBuf<int32_t> d_ladder_begin, d_rep_of_slot, d_pt_slot_of_rep;
    DevBuf<double> d_T_slot, d_E_sum, d_E2_sum;
    DevBuf<unsigned long long> d_n_e, d_att, d_accn;
    DevBuf<uint64_t> d_round;
    std::map<std::pair<int, int>, std::pair<cudaGraphExec_t, int>> pt_graphs;  // (n_sweep, phase)
    uint64_t pt_sweeps_done = 0;
    // amplitudes kept by pc_ssf_forward_keep: the token handed out with them (0: none)
    uint64_t amp_token = 0, amp_serial = 0;
    // rounds in one persistent cooperative launch (pt_persistent.cu)
    bool pt_persistent = false;
    DevBuf<unsigned int> d_bar;                 // grid barrier state (pc::kBarrierWords)
    std::map<std::array<int, 3>, int> persist_cap;  // (iso, fused, threads) -> resident blocks
    int barrier_polls = kBarrierMaxPolls;       // bound of each grid-barrier wait (pc_set_wait_limit)

    // pinned host staging for the small per-call transfers (upstream scalars,
    // energies, gradient sums, the device error flag): one synchronisation per
    // call instead of one per pageable copy
    void* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    cudaError_t stage(size_t bytes) {
        if (bytes <= h_stage_bytes) return cudaSuccess;
        if (h_stage) cudaFreeHost(h_stage);
        h_stage = nullptr;
        h_stage_bytes = 0;
        const cudaError_t e = cudaMallocHost(&h_stage, bytes);
        if (e == cudaSuccess) h_stage_bytes = bytes;
        return e;
    }

    // second stream for pc_step_host's result copy, which runs concurrently with
    // the last S(q) sample and the energy (they read the spins, never write them)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_swept = nullptr;

    ~pc_system() {
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (ev_swept) cudaEventDestroy(ev_swept);
        if (h_stage) cudaFreeHost(h_stage);
        for (auto& g : sweep_graphs) cudaGraphExecDestroy(g.second.first);
        for (auto& g : pt_graphs) cudaGraphExecDestroy(g.second.first);
        for (auto& e : ev_pool) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        if (stream && own_stream) cudaStreamDestroy(stream);
        d_reps.release();
        d_spins.release();
        d_T.release();
        d_Tq.release();
        d_sweep.release();
        d_acc.release();
        d_err.release();
        d_stage3.release();
        d_tab_active.release();
        d_tab_full.release();
        for (auto& t : d_colour_tiles) t.release();
        d_all_tiles.release();
        d_all_order.release();
        d_tile_begin.release();
        d_tile_end.release();
        d_partial.release();
        d_cell_tiles.release();
        d_cell_begin.release();
        d_cell_end.release();
        d_cell_partial.release();
        d_e.release();
        d_mag.release();
        d_theta.release();
        d_field.release();
        d_ssf_sum.release();
        d_ssf_sq.release();
        d_grad_g.release();
        d_grad_ones.release();
        d_group_partial.release();
        d_group_out.release();
        d_grad_out.release();
        d_grad_items.release();
        d_item_begin.release();
        d_item_end.release();
        d_grad_partial.release();
        for (auto& g : groups) {
            g.d_rep_index.release();
            g.d_sel_index.release();
            g.d_G.release();
            g.d_amp.release();
        }
        d_slot_of_rep.release();
        d_bar.release();
        d_ladder_begin.release();
        d_rep_of_slot.release();
        d_pt_slot_of_rep.release();
        d_T_slot.release();
        d_E_sum.release();
        d_E2_sum.release();
        d_n_e.release();
        d_att.release();
        d_accn.release();
        d_round.release();
    }

    int64_t Nc(int r) const { return int64_t(L[size_t(r)]) * L[size_t(r)] * L[size_t(r)]; }
    int64_t N(int r) const { return 16 * Nc(r); }

    void drop_graphs() {
        for (auto& g : sweep_graphs) cudaGraphExecDestroy(g.second.first);
        sweep_graphs.clear();
        for (auto& g : pt_graphs) cudaGraphExecDestroy(g.second.first);
        pt_graphs.clear();
    }
};

namespace {

int check_sys(pc_system* s, bool need_ready = true) {
    if (!s) return fail(PC_ERR_INVALID, "null system");
    if (need_ready && !s->ready) return fail(PC_ERR_STATE, "setup_lattice() has not been called");
    return PC_OK;
}
int check_rep(pc_system* s, int r) {
    if (r < 0 || r >= s->R) return fail(PC_ERR_INVALID, "replica index out of range");
    return PC_OK;
}

// Builds the structured shells of every sublattice for one table kind:
// identical to setup_lattice's split (src/MC.cpp:28-50): for each spec, the
// neighbours where this site's pyro_sl <= the other's form a shell applying J,
// the rest a shell applying J^T. keep_zero=false drops shells whose matrix is
// all zero (they contribute exactly nothing to the field).
int build_tables(pc_system* s, bool keep_zero, SlTable* out) {
    for (int sl = 0; sl < 16; ++sl) {
        SlTable& t = out[sl];
        std::memset(&t, 0, sizeof(t));
        const int p = sl % 4;
        const auto r = r_sl(sl);
        for (size_t c = 0; c < s->specs.size(); ++c) {
            const Coupling& cp = s->specs[c];
            std::vector<NbEntry> side[2];
            for (const auto& v : cp.rel[p]) {
                const std::array<int64_t, 3> x = {r[0] + v[0], r[1] + v[1], r[2] + v[2]};
                const int sl2 = sl_at(x);
                if (sl2 < 0) return fail(PC_ERR_INVALID, "coupling " + cp.name + ": displacement does not land on a site");
                const auto r2 = r_sl(sl2);
                NbEntry e;
                int64_t d[3];
                for (int a = 0; a < 3; ++a) {
                    d[a] = (x[a] - r2[a]) / 8;
                    if (d[a] < -1 || d[a] > 1)
                        return fail(PC_ERR_UNSUPPORTED, "coupling " + cp.name + ": reaches beyond the adjacent cubic cell");
                }
                e.dx = int8_t(d[0]);
                e.dy = int8_t(d[1]);
                e.dz = int8_t(d[2]);
                e.sl = uint8_t(sl2);
                side[(p <= sl2 % 4) ? 0 : 1].push_back(e);
            }
            for (int k = 0; k < 2; ++k) {
                if (side[k].empty()) continue;
                const double* M = k == 0 ? cp.J : cp.Jt;
                bool zero = true;
                for (int i = 0; i < 9; ++i) zero = zero && (M[i] == 0.0);
                if (zero && !keep_zero) continue;
                if (t.n_shell >= pc::kMaxShell || t.n_nb + int(side[k].size()) > pc::kMaxNb)
                    return fail(PC_ERR_UNSUPPORTED, "too many bond shells or neighbours per sublattice");
                for (const auto& e : side[k]) t.nb[t.n_nb++] = e;
                t.shell_end[t.n_shell] = t.n_nb;
                t.shell_spec[t.n_shell] = int(c) + (k == 1 ? 1000 : 0);
                for (int i = 0; i < 9; ++i) t.J[t.n_shell][i] = float(M[i]);
                t.n_shell++;
            }
        }
    }
    return PC_OK;
}

// Maps the coupling specs onto the structural neighbour groups of
// pyro_struct.cuh: for every sublattice and each of its 30 structural
// neighbours, the effective matrix is the sum over specs containing that
// displacement of J (source side) or J^T (target side), exactly the matrices
// setup_lattice would attach. If every spec displacement is structural and
// each group carries one matrix, the structured kernels apply.
void build_struct(pc_system* s) {
    s->structured = !s->force_generic;
    // the structured kernels address a replica's spins with unsigned 32-bit
    // byte offsets: 16 sublattices x Nc cells x 16 B must stay below 4 GB
    for (int r = 0; r < s->R; ++r)
        if (256.0 * double(s->Nc(r)) >= 4294967296.0) s->structured = false;
    s->grad_struct = s->structured && s->specs.size() <= 32;
    bool iso_nz[pc::kGroups], zero[pc::kGroups];  // per group, over all sublattices
    for (int g = 0; g < pc::kGroups; ++g) iso_nz[g] = zero[g] = true;
    std::memset(&s->mats, 0, sizeof(s->mats));
    std::memset(s->spec_mask, 0, sizeof(s->spec_mask));
    for (int sl = 0; sl < 16 && s->structured; ++sl) {
        const pc::SStruct T = pc::make_struct(sl);
        const int p = sl % 4;
        const auto r = r_sl(sl);
        double E[pc::kStructNb][9] = {};
        uint32_t owners[pc::kStructNb] = {};  // specs owning each structural displacement
        for (size_t ci = 0; ci < s->specs.size(); ++ci) {
            const Coupling& c = s->specs[ci];
            for (const auto& v : c.rel[p]) {
                const int g = pc::cs_group(sl, int(v[0]), int(v[1]), int(v[2]));
                if (std::llabs(v[0]) > 4 || std::llabs(v[1]) > 4 || std::llabs(v[2]) > 4 || g < 0) {
                    s->structured = false;
                    break;
                }
                const std::array<int64_t, 3> x = {r[0] + v[0], r[1] + v[1], r[2] + v[2]};
                const int sl2 = sl_at(x);
                int e = -1;
                for (int k = 0; k < pc::kStructNb; ++k) {
                    const auto r2 = r_sl(T.nb[k].sl);
                    if (T.nb[k].sl == sl2 && 8 * T.nb[k].dx + r2[0] == x[0] && 8 * T.nb[k].dy + r2[1] == x[1] &&
                        8 * T.nb[k].dz + r2[2] == x[2])
                        e = k;
                }
                if (e < 0) {
                    s->structured = false;
                    break;
                }
                const double* M = (p <= sl2 % 4) ? c.J : c.Jt;
                for (int i = 0; i < 9; ++i) E[e][i] += M[i];
                if (ci < 32) owners[e] |= 1u << ci;
            }
            if (!s->structured) break;
        }
        if (!s->structured) break;
        // the structured gradient needs one owner set per (group, bond side)
        for (int g = 0; g < pc::kGroups; ++g)
            for (int side = 0; side < 2; ++side) {
                bool first = true;
                for (int k = T.gbegin[g]; k < T.gbegin[g + 1]; ++k) {
                    if ((p <= T.nb[k].sl % 4 ? 0 : 1) != side) continue;
                    if (first) s->spec_mask[sl][g][side] = owners[k];
                    else if (s->spec_mask[sl][g][side] != owners[k]) s->grad_struct = false;
                    first = false;
                }
            }
        for (int g = 0; g < pc::kGroups; ++g) {
            const int b = T.gbegin[g], e1 = T.gbegin[g + 1];
            bool nonzero = false;
            for (int k = b; k < e1; ++k)
                for (int i = 0; i < 9; ++i) {
                    if (E[k][i] != E[b][i]) s->structured = false;
                    nonzero = nonzero || E[k][i] != 0.0;
                }
            for (int i = 0; i < 9; ++i) s->mats.M[sl][g][i] = float(E[b][i]);
            if (nonzero) s->mats.active[sl] |= 1u << g;
            const float* m = s->mats.M[sl][g];
            if (!(m[1] == 0.f && m[2] == 0.f && m[3] == 0.f && m[5] == 0.f && m[6] == 0.f && m[7] == 0.f &&
                  m[4] == m[0] && m[8] == m[0] && m[0] != 0.f))
                iso_nz[g] = false;
            if (nonzero) zero[g] = false;
        }
    }
    s->grad_struct = s->grad_struct && s->structured;
    bool others = true;  // every group but J2 (group 3) isotropic and nonzero
    for (int g = 0; g < pc::kGroups; ++g)
        if (g != 3) others = others && iso_nz[g];
    s->iso_kind = !s->structured ? 0 : (others && iso_nz[3]) ? 1 : (others && zero[3]) ? 2 : 0;
    s->iso_uniform = s->iso_kind != 0;
    for (int sl = 1; sl < 16; ++sl)
        for (int g = 0; g < pc::kGroups; ++g)
            if (s->mats.M[sl][g][0] != s->mats.M[0][g][0]) s->iso_uniform = false;
}

// Colour classes from the active bonds: sublattices joined by a nonzero bond
// never share a class. Greedy in sublattice order, at most 4 sublattices per
// class. With J1/J2 only this yields the 4 pyro_sl classes; J3 (which joins
// equal pyro_sl) refines them to the 16 conventional sublattices.
int build_colours(pc_system* s) {
    bool conflict[16][16] = {};
    for (int sl = 0; sl < 16; ++sl)
        for (int e = 0; e < s->tab_active[sl].n_nb; ++e) {
            const int o = s->tab_active[sl].nb[e].sl;
            conflict[sl][o] = conflict[o][sl] = true;
        }
    for (int sl = 0; sl < 16; ++sl)
        if (conflict[sl][sl])
            return fail(PC_ERR_UNSUPPORTED, "a coupling joins a sublattice to itself; sublattice colouring is not valid");
    s->colour_sls.clear();
    if (s->colouring == 0) {
        for (int sl = 0; sl < 16; ++sl) {
            s->colour_sls.push_back({sl});
            s->colour_of_sl[sl] = sl;
        }
        s->n_colours = 16;
        return PC_OK;
    }
    for (int sl = 0; sl < 16; ++sl) {
        int c = 0;
        for (; c < int(s->colour_sls.size()); ++c) {
            bool ok = s->colour_sls[size_t(c)].size() < 4;
            for (int o : s->colour_sls[size_t(c)]) ok = ok && !conflict[sl][o];
            if (ok) break;
        }
        if (c == int(s->colour_sls.size())) s->colour_sls.emplace_back();
        s->colour_sls[size_t(c)].push_back(sl);
        s->colour_of_sl[sl] = c;
    }
    s->n_colours = int(s->colour_sls.size());
    return PC_OK;
}

// Load variant 3 (row tiles staged into shared memory by bulk copies): the
// structured kernels, a whole x-row per tile (L <= threads <= 256).
bool use_staged(const pc_system* s) {
    if (!s->structured || s->load_variant != 3 || s->threads > 256) return false;
    for (int L : s->L)
        if (L > s->threads) return false;
    return true;
}

int build_tiles(pc_system* s) {
    const int T = s->threads;
    for (auto& t : s->d_colour_tiles) t.release();
    s->d_colour_tiles.clear();
    s->n_colour_tiles.clear();
    s->d_colour_tiles.resize(size_t(s->n_colours));
    const bool staged = use_staged(s);
    s->staged_rl = 0;
    for (int c = 0; c < s->n_colours; ++c) {
        std::vector<Tile> tiles;
        const auto& sls = s->colour_sls[size_t(c)];
        for (int r = 0; r < s->R; ++r)
            for (size_t k = 0; k < sls.size(); ++k) {
                const int L = s->L[size_t(r)];
                if (staged) {
                    // row tiles (x = replica, y = class slot << 8 | sublattice,
                    // z = first row cy0 + L cz, w = rows R): R*L <= T sites
                    const int R = std::max(1, std::min(L, T / L));
                    for (int cz = 0; cz < L; ++cz)
                        for (int cy0 = 0; cy0 < L; cy0 += R) {
                            const int n = std::min(R, L - cy0);
                            tiles.push_back(make_int4(r, int(k << 8) | sls[k], cy0 + L * cz, n));
                            s->staged_rl = std::max(s->staged_rl, n * L);
                        }
                    continue;
                }
                for (int64_t c0 = 0; c0 < s->Nc(r); c0 += T)
                    tiles.push_back(make_int4(r, int(k << 8) | sls[k], int(c0), int(std::min<int64_t>(T, s->Nc(r) - c0))));
            }
        PC_CK(s->d_colour_tiles[size_t(c)].alloc(tiles.size()));
        PC_CK(cudaMemcpy(s->d_colour_tiles[size_t(c)].p, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice));
        s->n_colour_tiles.push_back(int(tiles.size()));
    }
    std::vector<Tile> all;
    s->tile_begin.assign(size_t(s->R), 0);
    s->tile_end.assign(size_t(s->R), 0);
    for (int r = 0; r < s->R; ++r) {
        s->tile_begin[size_t(r)] = int(all.size());
        for (int sl = 0; sl < 16; ++sl)
            for (int64_t c0 = 0; c0 < s->Nc(r); c0 += T)
                all.push_back(make_int4(r, sl, int(c0), int(std::min<int64_t>(T, s->Nc(r) - c0))));
        s->tile_end[size_t(r)] = int(all.size());
    }
    s->n_all_tiles = int(all.size());
    PC_CK(s->d_all_tiles.alloc(all.size()));
    PC_CK(cudaMemcpy(s->d_all_tiles.p, all.data(), all.size() * sizeof(Tile), cudaMemcpyHostToDevice));
    std::vector<int32_t> order(all.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return all[size_t(x)].y < all[size_t(y)].y; });
    PC_CK(s->d_all_order.alloc(order.size()));
    PC_CK(cudaMemcpy(s->d_all_order.p, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    PC_CK(s->d_tile_begin.alloc(size_t(s->R)));
    PC_CK(s->d_tile_end.alloc(size_t(s->R)));
    PC_CK(cudaMemcpy(s->d_tile_begin.p, s->tile_begin.data(), sizeof(int32_t) * size_t(s->R), cudaMemcpyHostToDevice));
    PC_CK(cudaMemcpy(s->d_tile_end.p, s->tile_end.data(), sizeof(int32_t) * size_t(s->R), cudaMemcpyHostToDevice));
    // cell tiles of the per-cell energy kernel, replica by replica
    {
        std::vector<int4> ct;
        std::vector<int32_t> cb(size_t(s->R)), ce(size_t(s->R));
        for (int r = 0; r < s->R; ++r) {
            cb[size_t(r)] = int32_t(ct.size());
            for (int64_t c0 = 0; c0 < s->Nc(r); c0 += pc::kEnergyCellThreads)
                ct.push_back(make_int4(r, int(c0), int(std::min<int64_t>(pc::kEnergyCellThreads, s->Nc(r) - c0)), 0));
            ce[size_t(r)] = int32_t(ct.size());
        }
        s->n_cell_tiles = int(ct.size());
        PC_CK(s->d_cell_tiles.alloc(ct.size()));
        PC_CK(cudaMemcpy(s->d_cell_tiles.p, ct.data(), ct.size() * sizeof(int4), cudaMemcpyHostToDevice));
        PC_CK(s->d_cell_begin.alloc(size_t(s->R)));
        PC_CK(s->d_cell_end.alloc(size_t(s->R)));
        PC_CK(cudaMemcpy(s->d_cell_begin.p, cb.data(), sizeof(int32_t) * cb.size(), cudaMemcpyHostToDevice));
        PC_CK(cudaMemcpy(s->d_cell_end.p, ce.data(), sizeof(int32_t) * ce.size(), cudaMemcpyHostToDevice));
        PC_CK(s->d_cell_partial.alloc(ct.size() * 4));
    }
    // partial sums: energy (4 per tile) and gradient (4 + 9*n_spec per tile)
    const size_t width = size_t(4 + 9 * std::max<size_t>(1, s->specs.size()));
    PC_CK(s->d_partial.alloc(size_t(s->n_all_tiles) * width));
    // structured-gradient work items: runs of up to kGradK tiles of one
    // (replica, sublattice). Their partial-sum slots are replica-contiguous (the
    // per-replica finalize sums a slot range), but the items run sublattice by
    // sublattice: CTAs resident together then execute the same sublattice's
    // code, which keeps the instruction cache warm.
    std::vector<int4> items;
    s->item_begin.assign(size_t(s->R), 0);
    s->item_end.assign(size_t(s->R), 0);
    for (int r = 0; r < s->R; ++r) {
        s->item_begin[size_t(r)] = int(items.size());
        for (int t = s->tile_begin[size_t(r)]; t < s->tile_end[size_t(r)];) {
            int n = 1;
            while (n < pc::kGradK && t + n < s->tile_end[size_t(r)] && all[size_t(t + n)].y == all[size_t(t)].y) ++n;
            items.push_back(make_int4(t, n, int(items.size()), 0));  // z: partial-sum slot
            t += n;
        }
        s->item_end[size_t(r)] = int(items.size());
    }
    std::stable_sort(items.begin(), items.end(),
                     [&](const int4& x, const int4& y) { return all[size_t(x.x)].y < all[size_t(y.x)].y; });
    s->n_grad_items = int(items.size());
    PC_CK(s->d_grad_items.alloc(items.size()));
    PC_CK(cudaMemcpy(s->d_grad_items.p, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
    PC_CK(s->d_item_begin.alloc(size_t(s->R)));
    PC_CK(s->d_item_end.alloc(size_t(s->R)));
    PC_CK(cudaMemcpy(s->d_item_begin.p, s->item_begin.data(), sizeof(int32_t) * size_t(s->R), cudaMemcpyHostToDevice));
    PC_CK(cudaMemcpy(s->d_item_end.p, s->item_end.data(), sizeof(int32_t) * size_t(s->R), cudaMemcpyHostToDevice));
    PC_CK(s->d_grad_partial.alloc(items.size() * width));
    s->drop_graphs();
    return PC_OK;
}

pc::PassArgs pass_args(pc_system* s, int colour, uint64_t sweep_offset, int or_pass) {
    pc::PassArgs a;
    std::memset(&a, 0, sizeof(a));
    a.spins = s->d_spins.p;
    a.reps = s->d_reps.p;
    a.T_rep = s->d_T.p;
    a.Tq = s->d_Tq.p;
    a.sweep_base = s->d_sweep.p;
    a.sweep_offset = sweep_offset;
    a.seed = s->seed;
    a.rkeys = pc::philox_round_keys(s->seed);
    a.inv_T_ref = float(1.0 / s->T_ref);
    for (int i = 0; i < 3; ++i) a.B[i] = float(s->B[i]);
    a.tables = s->d_tab_active.p;
    const auto& sls = s->colour_sls[size_t(colour)];
    a.n_tab = int(sls.size());
    for (size_t k = 0; k < sls.size(); ++k) a.tab_sl[k] = sls[k];
    a.tiles = s->d_colour_tiles[size_t(colour)].p;
    a.n_tiles = s->n_colour_tiles[size_t(colour)];
    a.acc = s->d_acc.p;
    a.or_pass = or_pass;
    a.structured = s->structured ? 1 : 0;
    a.load_variant = use_staged(s) ? 3 : (s->load_variant == 3 ? 0 : s->load_variant);
    if (a.load_variant == 0 && s->iso_kind) a.load_variant = s->iso_kind == 1 ? pc::kVarIso : pc::kVarIsoNoJ2;
    a.mats = s->mats;
    a.staged_rl = s->staged_rl;
    a.err = s->d_err.p;
    a.wait_polls = s->wait_polls;
    return a;
}

// ctas_per_sm = 0: one CTA per tile (the hardware balances the waves)
int grid_for(pc_system* s, int n_tiles) {
    if (s->ctas_per_sm == 0) return std::max(1, n_tiles);
    return std::max(1, std::min(n_tiles, s->sms * s->ctas_per_sm));
}

// Launches one sweep's passes (sweep offset `off` relative to *d_sweep).
int enqueue_sweep(pc_system* s, uint64_t off, int n_or, bool record_events) {
    auto record = [&](int kind, bool start) -> int {
        if (!record_events) return PC_OK;
        if (start) {
            if (s->ev_used == s->ev_pool.size()) {
                cudaEvent_t a, b;
                PC_CK(cudaEventCreate(&a));
                PC_CK(cudaEventCreate(&b));
                s->ev_pool.push_back({a, b});
                s->ev_kind.push_back(kind);
            }
            s->ev_kind[s->ev_used] = kind;
            PC_CK(cudaEventRecord(s->ev_pool[s->ev_used].first, s->stream));
        } else {
            PC_CK(cudaEventRecord(s->ev_pool[s->ev_used].second, s->stream));
            s->ev_used++;
        }
        return PC_OK;
    };
    const bool fused = s->schedule == 1 && n_or >= 1 && s->update == 0;  // lifted sweeps: reference order
    const pc::PassMode mm = s->update == 1   ? pc::kLifted
                            : s->update == 2 ? pc::kLiftedRot
                            : fused ? (s->or_mode == 1 ? pc::kFusedReflect : pc::kFusedRotate)
                                    : pc::kMetropolis;
    for (int c = 0; c < s->n_colours; ++c) {
        const pc::PassArgs a = pass_args(s, c, off, 0);
        int rc = record(0, true);
        if (rc) return rc;
        pc::launch_colour_pass(mm, a, grid_for(s, a.n_tiles), s->threads, s->stream, s->pdl);
        PC_LAUNCH_CK();
        rc = record(0, false);
        if (rc) return rc;
        s->launches++;
    }
    const pc::PassMode om = s->or_mode == 1 ? pc::kOverrelaxReflect : pc::kOverrelaxRotate;
    for (int k = fused ? 1 : 0; k < n_or; ++k)
        for (int c = 0; c < s->n_colours; ++c) {
            const pc::PassArgs a = pass_args(s, c, off, k);
            int rc = record(1, true);
            if (rc) return rc;
            pc::launch_colour_pass(om, a, grid_for(s, a.n_tiles), s->threads, s->stream, s->pdl);
            PC_LAUNCH_CK();
            rc = record(1, false);
            if (rc) return rc;
            s->launches++;
        }
    return PC_OK;
}

// A captured graph of k sweeps (sweep offsets 0..k-1 from *d_sweep) plus one
// counter advance by k; nodes = kernels.
constexpr int kGraphSweeps = 16;
int sweep_graph(pc_system* s, int n_or, int k, cudaGraphExec_t* exec, int* nodes) {
    const auto key = std::make_pair(n_or, k);
    auto it = s->sweep_graphs.find(key);
    if (it != s->sweep_graphs.end()) {
        *exec = it->second.first;
        *nodes = it->second.second;
        return PC_OK;
    }
    const uint64_t before = s->launches;
    PC_CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = PC_OK;
    for (int i = 0; i < k && rc == PC_OK; ++i) rc = enqueue_sweep(s, uint64_t(i), n_or, false);
    pc::launch_advance_counter(s->d_sweep.p, uint64_t(k), s->stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        s->launches = before;
        return rc;
    }
    if (e != cudaSuccess) return fail(PC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(PC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    const int n = int(s->launches - before) + 1;
    s->launches = before;  // capture launched nothing
    s->sweep_graphs[key] = {x, n};
    *exec = x;
    *nodes = n;
    return PC_OK;
}

// Whether the sweeps of this system can run cluster-resident: the structured
// couplings, standard (not lifted) moves, all replicas of one size L <= 16,
// and the GPU able to hold a cluster of L CTAs with 16 L^2 float4 each.
bool cluster_eligible(pc_system* s, int n_or) {
    if (!s->structured || s->update != 0 || s->R < 1) return false;
    const int L = s->L[0];
    for (int r = 1; r < s->R; ++r)
        if (s->L[size_t(r)] != L) return false;
    if (L < 2 || L > 16) return false;
    const int fused = (s->schedule == 1 && n_or >= 1) ? 1 : 0;
    const std::array<int, 3> key = {L, fused, s->or_mode == 1 ? 1 : 0};
    auto it = s->cluster_cap.find(key);
    if (it == s->cluster_cap.end()) it = s->cluster_cap.emplace(key, pc::cluster_capacity(L, key[1], key[2])).first;
    return it->second > 0;
}

int launch_cluster(pc_system* s, int n_sweeps, int n_or) {
    pc::ClusterArgs a;
    std::memset(&a, 0, sizeof(a));
    a.spins = s->d_spins.p;
    a.reps = s->d_reps.p;
    a.T_rep = s->d_T.p;
    a.sweep_base = s->d_sweep.p;
    a.seed = s->seed;
    a.inv_T_ref = float(1.0 / s->T_ref);
    for (int i = 0; i < 3; ++i) a.B[i] = float(s->B[i]);
    a.acc = s->d_acc.p;
    a.mats = s->mats;
    a.L = s->L[0];
    a.n_sweeps = n_sweeps;
    a.n_or = n_or;
    a.fused = (s->schedule == 1 && n_or >= 1) ? 1 : 0;
    a.reflect = s->or_mode == 1 ? 1 : 0;
    a.n_classes = s->n_colours;
    for (int c = 0; c < s->n_colours; ++c) {
        const auto& sls = s->colour_sls[size_t(c)];
        a.class_n[c] = int(sls.size());
        for (size_t k = 0; k < sls.size(); ++k) a.class_sl[c][k] = sls[k];
    }
    pc::launch_cluster_sweeps(a, s->R, s->stream);
    PC_LAUNCH_CK();
    pc::launch_advance_counter(s->d_sweep.p, uint64_t(n_sweeps), s->stream);
    PC_LAUNCH_CK();
    s->launches += 2;
    return PC_OK;
}

// d_Tq from d_T (every writer of the temperatures but the exchange round,
// which updates both, comes before a batch of sweeps)
int refresh_tq(pc_system* s) {
    pc::launch_refresh_tq(s->d_T.p, s->d_Tq.p, s->R, float(1.0 / s->T_ref), s->stream);
    PC_LAUNCH_CK();
    s->launches++;
    return PC_OK;
}

int run_sweeps(pc_system* s, int n_sweeps, int n_or) {
    if (n_sweeps > 0) {
        const int rc = refresh_tq(s);
        if (rc) return rc;
    }
    if (s->cluster_sweep && !s->timing && n_sweeps > 0 && cluster_eligible(s, n_or)) {
        const int rc = launch_cluster(s, n_sweeps, n_or);
        if (rc) return rc;
        s->host_sweep += uint64_t(n_sweeps);
        return PC_OK;
    }
    if (s->timing) {
        for (int i = 0; i < n_sweeps; ++i) {
            int rc = enqueue_sweep(s, uint64_t(i), n_or, true);
            if (rc) return rc;
        }
        pc::launch_advance_counter(s->d_sweep.p, uint64_t(n_sweeps), s->stream);
        PC_LAUNCH_CK();
        s->launches++;
    } else {
        int done = 0;
        while (done < n_sweeps) {
            const int k = std::min(kGraphSweeps, n_sweeps - done);
            cudaGraphExec_t g;
            int nodes;
            int rc = sweep_graph(s, n_or, k, &g, &nodes);
            if (rc) return rc;
            PC_CK(cudaGraphLaunch(g, s->stream));
            s->launches += uint64_t(nodes);
            done += k;
        }
    }
    s->host_sweep += uint64_t(n_sweeps);
    return PC_OK;
}

// groups (iso_kind 1, iso_uniform): also the per-replica bare sums of S_i.S_j
// per coupling group into d_group_out [R][kGroups]
int enqueue_energy(pc_system* s, bool groups = false) {
    if (s->structured) {  // one thread per cubic cell, each bond once (energy_cell.cu)
        pc::EnergyCellArgs c;
        c.spins = s->d_spins.p;
        c.reps = s->d_reps.p;
        c.tiles = s->d_cell_tiles.p;
        c.n_tiles = s->n_cell_tiles;
        for (int i = 0; i < 3; ++i) c.B[i] = float(s->B[i]);
        c.partial = s->d_cell_partial.p;
        c.iso = s->iso_kind;
        c.uniform = s->iso_uniform ? 1 : 0;
        c.mats = s->mats;
        c.group_partial = nullptr;
        if (groups) {
            if (s->d_group_partial.n != size_t(s->n_cell_tiles) * pc::kGroups)
                PC_CK(s->d_group_partial.alloc(size_t(s->n_cell_tiles) * pc::kGroups));
            if (s->d_group_out.n != size_t(s->R) * pc::kGroups) PC_CK(s->d_group_out.alloc(size_t(s->R) * pc::kGroups));
            c.group_partial = s->d_group_partial.p;
        }
        pc::launch_energy_cells(c, s->stream);
        PC_LAUNCH_CK();
        pc::launch_energy_finalize(s->d_cell_partial.p, s->d_cell_begin.p, s->d_cell_end.p, s->d_reps.p, s->R,
                                   s->d_e.p, s->d_mag.p, s->stream);
        PC_LAUNCH_CK();
        s->launches += 2;
        if (groups) {
            pc::launch_grad_finalize(s->d_group_partial.p, pc::kGroups, s->d_cell_begin.p, s->d_cell_end.p, s->R,
                                     s->d_group_out.p, s->stream);
            PC_LAUNCH_CK();
            s->launches++;
        }
        return PC_OK;
    }
    pc::EnergyArgs a;
    a.spins = s->d_spins.p;
    a.reps = s->d_reps.p;
    a.tables = s->d_tab_active.p;
    a.tiles = s->d_all_tiles.p;
    a.order = s->d_all_order.p;
    a.n_tiles = s->n_all_tiles;
    for (int i = 0; i < 3; ++i) a.B[i] = float(s->B[i]);
    a.partial = s->d_partial.p;
    a.structured = s->structured ? 1 : 0;
    a.iso = s->iso_kind;
    a.mats = s->mats;
    pc::launch_energy_partials(a, s->threads, s->stream);
    PC_LAUNCH_CK();
    pc::launch_energy_finalize(s->d_partial.p, s->d_tile_begin.p, s->d_tile_end.p, s->d_reps.p, s->R, s->d_e.p,
                               s->d_mag.p, s->stream);
    PC_LAUNCH_CK();
    s->launches += 2;
    return PC_OK;
}

int enqueue_ssf(pc_system* s, const pc::SsfOut& o, bool selected_only) {
    for (auto& g : s->groups) {
        pc::SsfGeom geom;
        geom.L = g.L;
        geom.P = g.P;
        geom.Q = g.Q;
        geom.resolved = s->ssf_resolved ? 1 : 0;
        if (selected_only) {
            if (g.n_sel == 0) continue;
            geom.n_rep = g.n_sel;
            geom.rep_index = g.d_sel_index.p;
        } else {
            geom.n_rep = int(g.reps.size());
            geom.rep_index = g.d_rep_index.p;
        }
        pc::launch_ssf_xy(geom, s->d_spins.p, s->d_reps.p, g.d_G.p, s->stream);
        PC_LAUNCH_CK();
        pc::launch_ssf_z(geom, g.d_G.p, o, s->stream);
        PC_LAUNCH_CK();
        s->launches += 2;
    }
    return PC_OK;
}

pc::SsfOut ssf_out_base(pc_system* s) {
    pc::SsfOut o;
    std::memset(&o, 0, sizeof(o));
    o.n_corr = s->n_corr;
    for (int c = 0; c < s->n_corr; ++c) {
        o.corr_a[c] = s->corr_a[c];
        o.corr_b[c] = s->corr_b[c];
    }
    o.slot_stride = s->slot_stride;
    return o;
}

int ensure_groups(pc_system* s) {
    if (!s->groups.empty()) return PC_OK;
    std::map<int, std::vector<int>> by_L;
    for (int r = 0; r < s->R; ++r) by_L[s->L[size_t(r)]].push_back(r);
    for (auto& kv : by_L) {
        SsfGroup g;
        g.L = kv.first;
        split_PQ(g.L, &g.P, &g.Q);
        if (9 * g.L + 3 * g.L * g.L > 200 * 1024 / 8)
            return fail(PC_ERR_UNSUPPORTED, "SSF supports L up to 90 (one z plane per CTA in shared memory)");
        g.reps = kv.second;
        s->groups.push_back(std::move(g));
    }
    pc::ssf_prepare();
    for (auto& g : s->groups) {
        PC_CK(g.d_sel_index.alloc(g.reps.size()));
        PC_CK(g.d_rep_index.alloc(g.reps.size()));
        PC_CK(cudaMemcpy(g.d_rep_index.p, g.reps.data(), sizeof(int32_t) * g.reps.size(), cudaMemcpyHostToDevice));
        const size_t L3 = size_t(g.L) * g.L * g.L;
        PC_CK(g.d_G.alloc(g.reps.size() * 48 * L3));  // 3 components x 8 half-groups, or x 16 sublattices
    }
    return PC_OK;
}

}  // namespace

extern "C" {

const char* pc_last_error(void) { return g_last_error.c_str(); }
int pc_version(void) { return 100; }

int pc_create(int n_replicas, const int32_t* L, uint64_t seed, pc_system** out) {
    if (!out) return fail(PC_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (n_replicas <= 0 || !L) return fail(PC_ERR_INVALID, "need at least one replica");
    for (int r = 0; r < n_replicas; ++r)
        if (L[r] < 1 || L[r] > 1024) return fail(PC_ERR_INVALID, "L must be in [1, 1024]");
    auto* s = new pc_system();
    s->R = n_replicas;
    s->seed = seed;
    s->L.assign(L, L + n_replicas);
    s->off.resize(size_t(n_replicas));
    int64_t o = 0;
    for (int r = 0; r < n_replicas; ++r) {
        s->off[size_t(r)] = o;
        o += s->N(r);
    }
    s->N_tot = o;
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    std::vector<ReplicaDev> reps(static_cast<size_t>(n_replicas));
    for (int r = 0; r < n_replicas; ++r)
        reps[size_t(r)] = {L[r], int32_t(s->Nc(r)), s->off[size_t(r)], pc::fastdiv_magic(L[r])};
    if (e == cudaSuccess) e = s->d_reps.alloc(size_t(n_replicas));
    if (e == cudaSuccess) e = cudaMemcpy(s->d_reps.p, reps.data(), sizeof(ReplicaDev) * reps.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = s->d_spins.alloc(size_t(s->N_tot));
    if (e == cudaSuccess) e = cudaMemset(s->d_spins.p, 0, sizeof(float4) * size_t(s->N_tot));
    if (e == cudaSuccess) e = s->d_T.alloc(size_t(n_replicas));
    if (e == cudaSuccess) e = s->d_Tq.alloc(size_t(n_replicas));
    if (e == cudaSuccess) e = s->d_sweep.alloc(1);
    if (e == cudaSuccess) e = cudaMemset(s->d_sweep.p, 0, sizeof(uint64_t));
    if (e == cudaSuccess) e = s->d_acc.alloc(size_t(n_replicas));
    if (e == cudaSuccess) e = s->d_err.alloc(1);
    if (e == cudaSuccess) e = cudaMemset(s->d_err.p, 0, sizeof(int));
    if (e == cudaSuccess) e = s->d_e.alloc(size_t(n_replicas));
    if (e == cudaSuccess) e = s->d_mag.alloc(size_t(3 * n_replicas));
    if (e != cudaSuccess) {
        delete s;
        return fail(PC_ERR_CUDA, std::string("pc_create: ") + cudaGetErrorString(e));
    }
    *out = s;
    return PC_OK;
}

int pc_destroy(pc_system* sys) {
    if (!sys) return PC_OK;
    if (sys->stream) cudaStreamSynchronize(sys->stream);
    delete sys;
    return PC_OK;
}

int pc_set_stream(pc_system* sys, void* stream) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (stream == nullptr || stream == cudaStreamLegacy || stream == cudaStreamPerThread)
        return fail(PC_ERR_INVALID, "pc_set_stream needs a created stream (the default stream cannot be captured)");
    PC_CK(cudaStreamSynchronize(sys->stream));
    if (sys->own_stream) cudaStreamDestroy(sys->stream);
    sys->stream = static_cast<cudaStream_t>(stream);
    sys->own_stream = false;
    sys->drop_graphs();
    return PC_OK;
}

int pc_set_seed(pc_system* sys, uint64_t seed) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    sys->seed = seed;
    sys->drop_graphs();
    return PC_OK;
}

int pc_define_coupling(pc_system* sys, const char* name, const int64_t* rel_vecs, const int32_t* n_rel, const double* J) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (!name || !n_rel || !J) return fail(PC_ERR_INVALID, "null argument");
    for (const auto& c : sys->specs)
        if (c.name == name) return fail(PC_ERR_INVALID, "Coupling names must be unique");
    if (sys->ready) return fail(PC_ERR_STATE, "couplings must be defined before setup_lattice()");
    Coupling c;
    c.name = name;
    size_t k = 0;
    for (int p = 0; p < 4; ++p) {
        if (n_rel[p] < 0) return fail(PC_ERR_INVALID, "negative displacement count");
        for (int j = 0; j < n_rel[p]; ++j, ++k)
            c.rel[p].push_back({rel_vecs[3 * k], rel_vecs[3 * k + 1], rel_vecs[3 * k + 2]});
    }
    for (int i = 0; i < 9; ++i) c.J[i] = J[i];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) c.Jt[3 * a + b] = J[3 * b + a];
    sys->specs.push_back(std::move(c));
    return PC_OK;
}

int pc_set_coupling_matrix(pc_system* sys, int spec, const double* J) {
    return pc_set_coupling_matrices(sys, 1, &spec, J);
}

int pc_set_coupling_matrices(pc_system* sys, int n, const int32_t* specs, const double* J) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!specs || !J))) return fail(PC_ERR_INVALID, "null specs or matrices");
    bool changed = false;
    for (int k = 0; k < n; ++k) {
        if (specs[k] < 0 || specs[k] >= int(sys->specs.size())) return fail(PC_ERR_INVALID, "spec index out of range");
        for (int i = 0; i < 9; ++i) changed = changed || sys->specs[size_t(specs[k])].J[i] != J[9 * k + i];
    }
    // the tables, colour classes and structure follow the matrices alone
    if (!changed) return PC_OK;
    for (int k = 0; k < n; ++k) {
        Coupling& c = sys->specs[size_t(specs[k])];
        const double* Jk = J + 9 * k;
        for (int i = 0; i < 9; ++i) c.J[i] = Jk[i];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) c.Jt[3 * a + b] = Jk[3 * b + a];
    }
    rc = build_tables(sys, false, sys->tab_active);
    if (rc) return rc;
    rc = build_tables(sys, true, sys->tab_full);
    if (rc) return rc;
    const int old_colours = sys->n_colours;
    rc = build_colours(sys);
    if (rc) return rc;
    build_struct(sys);
    PC_CK(cudaStreamSynchronize(sys->stream));
    PC_CK(cudaMemcpy(sys->d_tab_active.p, sys->tab_active, sizeof(SlTable) * 16, cudaMemcpyHostToDevice));
    PC_CK(cudaMemcpy(sys->d_tab_full.p, sys->tab_full, sizeof(SlTable) * 16, cudaMemcpyHostToDevice));
    if (sys->colouring != 0 || old_colours != sys->n_colours) return build_tiles(sys);
    sys->drop_graphs();
    return PC_OK;
}

int pc_set_global_field(pc_system* sys, const double* B3) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (sys->B[0] == B3[0] && sys->B[1] == B3[1] && sys->B[2] == B3[2]) return PC_OK;
    for (int i = 0; i < 3; ++i) sys->B[i] = B3[i];
    sys->drop_graphs();
    return PC_OK;
}
int pc_get_global_field(pc_system* sys, double* B3) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    for (int i = 0; i < 3; ++i) B3[i] = sys->B[i];
    return PC_OK;
}
int pc_set_T_ref(pc_system* sys, double T_ref) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (!(T_ref > 0)) return fail(PC_ERR_INVALID, "T_ref must be positive");
    sys->T_ref = T_ref;
    sys->drop_graphs();
    return PC_OK;
}
int pc_set_overrelax_mode(pc_system* sys, int mode) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (mode != 0 && mode != 1) return fail(PC_ERR_INVALID, "overrelaxation mode must be 0 (rotation) or 1 (reflection)");
    sys->or_mode = mode;
    sys->drop_graphs();
    return PC_OK;
}

int pc_set_sweep_schedule(pc_system* sys, int schedule) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (schedule != 0 && schedule != 1) return fail(PC_ERR_INVALID, "sweep schedule must be 0 (reference order) or 1 (fused)");
    sys->schedule = schedule;
    sys->drop_graphs();
    return PC_OK;
}

int pc_set_update(pc_system* sys, int mode) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (mode < 0 || mode > 2)
        return fail(PC_ERR_INVALID, "update must be 0 (Metropolis), 1 (lifted) or 2 (lifted, rotation form)");
    sys->update = mode;
    sys->drop_graphs();
    return PC_OK;
}

int pc_set_launch_overlap(pc_system* sys, int on) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    sys->pdl = on != 0;
    sys->drop_graphs();
    return PC_OK;
}

int pc_set_cluster_sweeps(pc_system* sys, int on) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (on && !cluster_eligible(sys, 1))
        return fail(PC_ERR_UNSUPPORTED, "cluster-resident sweeps need the structured pyrochlore couplings, standard "
                                        "moves and replicas of one size L <= 16 that fit a thread-block cluster");
    sys->cluster_sweep = on != 0;
    return PC_OK;
}
int pc_get_cluster_sweeps(pc_system* sys, int* on) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    *on = sys->cluster_sweep ? 1 : 0;
    return PC_OK;
}

int pc_set_kernel_path(pc_system* sys, int force_generic) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    sys->force_generic = force_generic != 0;
    if (sys->ready) build_struct(sys);
    sys->drop_graphs();
    return PC_OK;
}

int pc_kernel_path(pc_system* sys, int* structured) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    *structured = sys->structured ? 1 : 0;
    return PC_OK;
}

int pc_set_colouring(pc_system* sys, int mode) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (sys->ready) return fail(PC_ERR_STATE, "colouring must be chosen before setup_lattice()");
    if (mode != 0 && mode != 1) return fail(PC_ERR_INVALID, "colouring mode must be 0 (per sublattice) or 1 (fewest classes)");
    sys->colouring = mode;
    return PC_OK;
}

int pc_setup_lattice(pc_system* sys) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (sys->ready) return fail(PC_ERR_STATE, "setup_lattice() already called");
    if (sys->specs.size() > 100) return fail(PC_ERR_UNSUPPORTED, "at most 100 coupling specs");
    rc = build_tables(sys, false, sys->tab_active);
    if (rc) return rc;
    rc = build_tables(sys, true, sys->tab_full);
    if (rc) return rc;
    rc = build_colours(sys);
    if (rc) return rc;
    build_struct(sys);
    PC_CK(sys->d_tab_active.alloc(16));
    PC_CK(sys->d_tab_full.alloc(16));
    PC_CK(cudaMemcpy(sys->d_tab_active.p, sys->tab_active, sizeof(SlTable) * 16, cudaMemcpyHostToDevice));
    PC_CK(cudaMemcpy(sys->d_tab_full.p, sys->tab_full, sizeof(SlTable) * 16, cudaMemcpyHostToDevice));
    rc = build_tiles(sys);
    if (rc) return rc;
    sys->ready = true;
    return PC_OK;
}

int pc_pyrochlore_displacements(int kind, int pyro_sl, int64_t* out, int max_n, int* n) {
    if (pyro_sl < 0 || pyro_sl > 3) return fail(PC_ERR_INVALID, "pyro_sl must be 0..3");
    const bool pair = kind >= 10 && kind <= 13;
    if (!pair && (kind < 1 || kind > 4)) return fail(PC_ERR_INVALID, "unknown displacement table kind");
    const int64_t r2 = (kind == 2) ? 24 : (kind == 1 || pair) ? 8 : 32;
    const std::array<int64_t, 3> x0 = {kLink[pyro_sl][0], kLink[pyro_sl][1], kLink[pyro_sl][2]};
    int cnt = 0;
    for (int64_t dx = -4; dx <= 4; ++dx)
        for (int64_t dy = -4; dy <= 4; ++dy)
            for (int64_t dz = -4; dz <= 4; ++dz) {
                if (dx * dx + dy * dy + dz * dz != r2) continue;
                const std::array<int64_t, 3> x = {x0[0] + dx, x0[1] + dy, x0[2] + dz};
                const int sl2 = sl_at(x);
                if (sl2 < 0) continue;
                if (kind == 3 || kind == 4) {
                    const bool mid = sl_at({x0[0] + dx / 2, x0[1] + dy / 2, x0[2] + dz / 2}) >= 0;
                    if ((kind == 3) != mid) continue;
                }
                if (pair && sl2 % 4 != kind - 10) continue;
                if (cnt >= max_n) return fail(PC_ERR_INVALID, "max_n too small");
                out[3 * cnt] = dx;
                out[3 * cnt + 1] = dy;
                out[3 * cnt + 2] = dz;
                ++cnt;
            }
    *n = cnt;
    return PC_OK;
}

int pc_num_replicas(pc_system* sys, int* n) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    *n = sys->R;
    return PC_OK;
}
int pc_num_spins(pc_system* sys, int replica, int64_t* n) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    *n = sys->N(replica);
    return PC_OK;
}
int pc_colours(pc_system* sys, int* n_colours, int32_t* colour_of_sl) {
    int rc = check_sys(sys);
    if (rc) return rc;
    *n_colours = sys->n_colours;
    if (colour_of_sl)
        for (int i = 0; i < 16; ++i) colour_of_sl[i] = sys->colour_of_sl[i];
    return PC_OK;
}

int pc_neighbour_table(pc_system* sys, int replica, int spec, int max_nb, int32_t* out) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    if (spec < 0 || spec >= int(sys->specs.size())) return fail(PC_ERR_INVALID, "spec index out of range");
    const Coupling& c = sys->specs[size_t(spec)];
    const int L = sys->L[size_t(replica)];
    const int64_t Nc = sys->Nc(replica);
    for (int p = 0; p < 4; ++p)
        if (int(c.rel[p].size()) > max_nb) return fail(PC_ERR_INVALID, "max_nb too small");
    for (int sl = 0; sl < 16; ++sl) {
        const auto r = r_sl(sl);
        const auto& rel = c.rel[sl % 4];
        for (int64_t cell = 0; cell < Nc; ++cell) {
            const int64_t cx = cell % L, cy = (cell / L) % L, cz = cell / (int64_t(L) * L);
            int32_t* row = out + (size_t(sl) * Nc + cell) * size_t(max_nb);
            for (int j = 0; j < max_nb; ++j) row[j] = -1;
            for (size_t j = 0; j < rel.size(); ++j) {
                const std::array<int64_t, 3> x = {8 * cx + r[0] + rel[j][0], 8 * cy + r[1] + rel[j][1],
                                                  8 * cz + r[2] + rel[j][2]};
                const int sl2 = sl_at(x);
                if (sl2 < 0) return fail(PC_ERR_INVALID, "displacement does not land on a site");
                const auto r2 = r_sl(sl2);
                const int64_t nx = pmod((x[0] - r2[0]) / 8, L), ny = pmod((x[1] - r2[1]) / 8, L),
                              nz = pmod((x[2] - r2[2]) / 8, L);
                row[j] = int32_t(int64_t(sl2) * Nc + nx + L * (ny + int64_t(L) * nz));
            }
        }
    }
    return PC_OK;
}

int pc_site_positions(pc_system* sys, int replica, int64_t* pos, int32_t* sl_out) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    const int L = sys->L[size_t(replica)];
    const int64_t Nc = sys->Nc(replica);
    for (int sl = 0; sl < 16; ++sl) {
        const auto r = r_sl(sl);
        for (int64_t cell = 0; cell < Nc; ++cell) {
            const int64_t c[3] = {cell % L, (cell / L) % L, cell / (int64_t(L) * L)};
            const size_t i = size_t(sl) * size_t(Nc) + size_t(cell);
            for (int a = 0; a < 3; ++a) pos[3 * i + a] = pmod(8 * c[a] + r[a], 8 * int64_t(L));
            if (sl_out) sl_out[i] = sl;
        }
    }
    return PC_OK;
}

int pc_launch_count(pc_system* sys, uint64_t* n) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    *n = sys->launches;
    return PC_OK;
}

int pc_set_spins(pc_system* sys, int replica, const double* S) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    const int64_t n = sys->N(replica);
    std::vector<float4> buf(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i)
        buf[size_t(i)] = make_float4(float(S[3 * i]), float(S[3 * i + 1]), float(S[3 * i + 2]), 0.f);
    PC_CK(cudaMemcpyAsync(sys->d_spins.p + sys->off[size_t(replica)], buf.data(), sizeof(float4) * size_t(n),
                          cudaMemcpyHostToDevice, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}
int pc_get_spins(pc_system* sys, int replica, double* S) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    const int64_t n = sys->N(replica);
    std::vector<float4> buf(static_cast<size_t>(n));
    PC_CK(cudaMemcpyAsync(buf.data(), sys->d_spins.p + sys->off[size_t(replica)], sizeof(float4) * size_t(n),
                          cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    for (int64_t i = 0; i < n; ++i) {
        S[3 * i] = buf[size_t(i)].x;
        S[3 * i + 1] = buf[size_t(i)].y;
        S[3 * i + 2] = buf[size_t(i)].z;
    }
    return PC_OK;
}
int pc_set_spins_f4(pc_system* sys, int replica, const float* S4) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    PC_CK(cudaMemcpyAsync(sys->d_spins.p + sys->off[size_t(replica)], S4, sizeof(float4) * size_t(sys->N(replica)),
                          cudaMemcpyHostToDevice, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}
int pc_get_spins_f4(pc_system* sys, int replica, float* S4) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    PC_CK(cudaMemcpyAsync(S4, sys->d_spins.p + sys->off[size_t(replica)], sizeof(float4) * size_t(sys->N(replica)),
                          cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}
int pc_random_spins(pc_system* sys, uint64_t seed) {
    int rc = check_sys(sys);
    if (rc) return rc;
    pc::launch_random_spins(sys->d_spins.p, sys->d_reps.p, sys->d_all_tiles.p, sys->n_all_tiles, seed, sys->threads,
                            sys->stream);
    PC_LAUNCH_CK();
    sys->launches++;
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}
int pc_spins_device(pc_system* sys, int replica, void** dev_ptr) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    *dev_ptr = sys->d_spins.p + sys->off[size_t(replica)];
    return PC_OK;
}
int pc_get_sweep_counter(pc_system* sys, int replica, uint64_t* sweep) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    PC_CK(cudaStreamSynchronize(sys->stream));
    PC_CK(cudaMemcpy(sweep, sys->d_sweep.p, sizeof(uint64_t), cudaMemcpyDeviceToHost));
    return PC_OK;
}
int pc_set_sweep_counter(pc_system* sys, int replica, uint64_t sweep) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    PC_CK(cudaStreamSynchronize(sys->stream));
    PC_CK(cudaMemcpy(sys->d_sweep.p, &sweep, sizeof(uint64_t), cudaMemcpyHostToDevice));
    sys->host_sweep = sweep;
    return PC_OK;
}

// The device error flag as read back (flag != 0: one of a kernel's bounded
// waits ran out): clears it and reports the failure.
int device_error_flag(pc_system* s, int flag) {
    if (!flag) return PC_OK;
    PC_CK(cudaMemsetAsync(s->d_err.p, 0, sizeof(int), s->stream));
    if (flag == pc::kErrGridBarrier)
        return fail(PC_ERR_TIMEOUT, "the persistent tempering kernel stopped waiting at a grid barrier (bounded wait "
                                    "ran out); the round was left unfinished");
    return fail(PC_ERR_TIMEOUT, "a colour pass stopped waiting for its staged neighbour rows (bounded wait ran out); "
                                "the updates of that pass were skipped");
}

// Reads (and clears) the device error flag. Synchronises the system's stream.
int device_error(pc_system* s) {
    int flag = 0;
    PC_CK(cudaMemcpyAsync(&flag, s->d_err.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    PC_CK(cudaStreamSynchronize(s->stream));
    return device_error_flag(s, flag);
}

int pc_sweep(pc_system* sys, const double* T, int n_sweeps, int n_overrelax, uint64_t* accepted) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!T) return fail(PC_ERR_INVALID, "null temperature array");
    if (n_sweeps < 0 || n_overrelax < 0 || n_overrelax > 200) return fail(PC_ERR_INVALID, "bad sweep counts");
    for (int r = 0; r < sys->R; ++r)
        if (!(T[r] > 0)) return fail(PC_ERR_INVALID, "temperatures must be positive");
    PC_CK(cudaMemcpyAsync(sys->d_T.p, T, sizeof(double) * size_t(sys->R), cudaMemcpyHostToDevice, sys->stream));
    PC_CK(cudaMemsetAsync(sys->d_acc.p, 0, sizeof(unsigned long long) * size_t(sys->R), sys->stream));
    rc = run_sweeps(sys, n_sweeps, n_overrelax);
    if (rc) return rc;
    if (accepted) {
        PC_CK(cudaMemcpyAsync(accepted, sys->d_acc.p, sizeof(uint64_t) * size_t(sys->R), cudaMemcpyDeviceToHost,
                              sys->stream));
        return device_error(sys);
    }
    return PC_OK;
}

int pc_overrelax_all(pc_system* sys) {
    int rc = check_sys(sys);
    if (rc) return rc;
    const pc::PassMode om = sys->or_mode == 1 ? pc::kOverrelaxReflect : pc::kOverrelaxRotate;
    for (int c = 0; c < sys->n_colours; ++c) {
        const pc::PassArgs a = pass_args(sys, c, 0, 0);
        pc::launch_colour_pass(om, a, grid_for(sys, a.n_tiles), sys->threads, sys->stream);
        PC_LAUNCH_CK();
        sys->launches++;
    }
    pc::launch_advance_counter(sys->d_sweep.p, 1, sys->stream);
    PC_LAUNCH_CK();
    sys->launches++;
    sys->host_sweep++;
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}

int pc_overrelax_theta(pc_system* sys, int replica, const double* theta) {
    int rc = check_sys(sys);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    const int64_t n = sys->N(replica);
    if (theta) {
        PC_CK(sys->d_theta.alloc(size_t(n)));
        PC_CK(cudaMemcpy(sys->d_theta.p, theta, sizeof(double) * size_t(n), cudaMemcpyHostToDevice));
    }
    for (int c = 0; c < sys->n_colours; ++c) {
        pc::PassArgs a = pass_args(sys, c, 0, 0);
        a.theta = sys->d_theta.p;
        a.theta_replica = replica;
        // only the requested replica's tiles: the theta array is per site of it
        std::vector<Tile> tiles;
        const auto& sls = sys->colour_sls[size_t(c)];
        for (size_t k = 0; k < sls.size(); ++k)
            for (int64_t c0 = 0; c0 < sys->Nc(replica); c0 += sys->threads)
                tiles.push_back(make_int4(replica, int(k << 8) | sls[k], int(c0),
                                          int(std::min<int64_t>(sys->threads, sys->Nc(replica) - c0))));
        DevBuf<Tile> dt;
        PC_CK(dt.alloc(tiles.size()));
        PC_CK(cudaMemcpy(dt.p, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice));
        a.tiles = dt.p;
        a.n_tiles = int(tiles.size());
        pc::launch_colour_pass(theta ? pc::kOverrelaxTheta : pc::kOverrelaxReflect, a, grid_for(sys, a.n_tiles),
                               sys->threads, sys->stream);
        PC_LAUNCH_CK();
        sys->launches++;
        PC_CK(cudaStreamSynchronize(sys->stream));
        dt.release();
    }
    return PC_OK;
}

int pc_energy(pc_system* sys, double* e_per_cell, double* mag) {
    int rc = check_sys(sys);
    if (rc) return rc;
    rc = enqueue_energy(sys);
    if (rc) return rc;
    const size_t R = size_t(sys->R);
    PC_CK(sys->stage(sizeof(double) * 4 * R + sizeof(int)));
    double* st = static_cast<double*>(sys->h_stage);
    int* flag = reinterpret_cast<int*>(st + 4 * R);
    PC_CK(cudaMemcpyAsync(st, sys->d_e.p, sizeof(double) * R, cudaMemcpyDeviceToHost, sys->stream));
    if (mag) PC_CK(cudaMemcpyAsync(st + R, sys->d_mag.p, sizeof(double) * 3 * R, cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaMemcpyAsync(flag, sys->d_err.p, sizeof(int), cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    std::memcpy(e_per_cell, st, sizeof(double) * R);
    if (mag) std::memcpy(mag, st + R, sizeof(double) * 3 * R);
    return device_error_flag(sys, *flag);
}

int pc_local_field(pc_system* sys, int replica, double* h) {
    int rc = check_sys(sys);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    if (sys->d_field.n != size_t(sys->N_tot)) PC_CK(sys->d_field.alloc(size_t(sys->N_tot)));
    pc::FieldArgs a;
    a.spins = sys->d_spins.p;
    a.reps = sys->d_reps.p;
    a.tables = sys->d_tab_active.p;
    a.tiles = sys->d_all_tiles.p + sys->tile_begin[size_t(replica)];
    a.n_tiles = sys->tile_end[size_t(replica)] - sys->tile_begin[size_t(replica)];
    a.h_out = sys->d_field.p;
    pc::launch_local_field(a, sys->threads, sys->stream);
    PC_LAUNCH_CK();
    sys->launches++;
    const int64_t n = sys->N(replica);
    std::vector<float4> buf(static_cast<size_t>(n));
    PC_CK(cudaMemcpyAsync(buf.data(), sys->d_field.p + sys->off[size_t(replica)], sizeof(float4) * size_t(n),
                          cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    for (int64_t i = 0; i < n; ++i) {
        h[3 * i] = buf[size_t(i)].x;
        h[3 * i + 1] = buf[size_t(i)].y;
        h[3 * i + 2] = buf[size_t(i)].z;
    }
    return PC_OK;
}

// ------------------------------------------------------------------- SSF
int pc_ssf_configure(pc_system* sys, const char* const* names, int n_corr, int n_slots, const int32_t* L_of_slot) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (n_corr < 1 || n_corr > 9) return fail(PC_ERR_INVALID, "ssf_manager: between 1 and 9 correlators");
    if (n_slots < 0) return fail(PC_ERR_INVALID, "negative slot count");
    // ssf_manager.hpp:176-193
    auto axis = [](char c) -> int { return c == 'x' ? 0 : c == 'y' ? 1 : c == 'z' ? 2 : -1; };
    for (int c = 0; c < n_corr; ++c) {
        const std::string nm = names[c] ? names[c] : "";
        if (nm.size() != 2) return fail(PC_ERR_INVALID, "ssf_manager: correlator name must be 2 chars: " + nm);
        for (int k = 0; k < 2; ++k)
            if (axis(nm[size_t(k)]) < 0)
                return fail(PC_ERR_INVALID, std::string("ssf_manager: unknown spin component '") + nm[size_t(k)] + "'");
        sys->corr_a[c] = axis(nm[0]);
        sys->corr_b[c] = axis(nm[1]);
    }
    rc = ensure_groups(sys);
    if (rc) return rc;
    sys->n_corr = n_corr;
    sys->n_slots = n_slots;
    sys->L_of_slot.assign(L_of_slot, L_of_slot + n_slots);
    int64_t max_nk = 1;
    for (int sl = 0; sl < n_slots; ++sl) {
        bool found = false;
        for (auto& g : sys->groups) found = found || (g.L == L_of_slot[sl]);
        if (!found) return fail(PC_ERR_INVALID, "slot size matches no replica");
        max_nk = std::max<int64_t>(max_nk, int64_t(L_of_slot[sl]) * L_of_slot[sl] * L_of_slot[sl]);
    }
    if (sys->ssf_resolved)
        for (auto& g : sys->groups)
            if (g.P > 8 || g.Q > 8)
                return fail(PC_ERR_UNSUPPORTED, "sublattice-resolved S(q) needs every L to factor into two parts <= 8");
    sys->slot_stride = int64_t(n_corr) * max_nk * 2 * (sys->ssf_resolved ? 256 : 1);
    PC_CK(sys->d_ssf_sum.alloc(size_t(std::max(1, n_slots)) * size_t(sys->slot_stride)));
    PC_CK(sys->d_ssf_sq.alloc(size_t(std::max(1, n_slots)) * size_t(sys->slot_stride)));
    PC_CK(cudaMemset(sys->d_ssf_sum.p, 0, sizeof(double) * sys->d_ssf_sum.n));
    PC_CK(cudaMemset(sys->d_ssf_sq.p, 0, sizeof(double) * sys->d_ssf_sq.n));
    PC_CK(sys->d_slot_of_rep.alloc(size_t(sys->R)));
    sys->ssf_n.assign(size_t(n_slots), 0);
    sys->ssf_ready = true;
    sys->drop_graphs();
    return PC_OK;
}

int pc_ssf_merge(pc_system* sys, const int32_t* slots, int K, double* static_corr, double* static_corr_2,
                 double* var_inter, double* var_intra, double* w, double* chi_frac, double* tr) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->ssf_ready) return fail(PC_ERR_STATE, "ssf not configured");
    if (sys->ssf_resolved) return fail(PC_ERR_UNSUPPORTED, "seed merge works on the contracted S(q)");
    if (K < 1 || !slots) return fail(PC_ERR_INVALID, "need at least one slot");
    const int L = sys->L_of_slot[size_t(slots[0])];
    uint64_t n = 0;
    for (int s = 0; s < K; ++s) {
        if (slots[s] < 0 || slots[s] >= sys->n_slots) return fail(PC_ERR_INVALID, "slot index out of range");
        if (sys->L_of_slot[size_t(slots[s])] != L) return fail(PC_ERR_INVALID, "slots differ in lattice size");
        const uint64_t ns = sys->ssf_n[size_t(slots[s])];
        if (s == 0) n = ns;
        if (ns != n) return fail(PC_ERR_INVALID, "seeds differ in their sample counts (the merge assumes one count)");
    }
    if (n == 0) return fail(PC_ERR_STATE, "no samples in the slots");
    pc::MergeArgs a;
    std::memset(&a, 0, sizeof(a));
    a.sum = sys->d_ssf_sum.p;
    a.sq = sys->d_ssf_sq.p;
    a.slot_stride = sys->slot_stride;
    a.K = K;
    a.n_corr = sys->n_corr;
    a.n_k = L * L * L;
    a.n = double(n);
    const int want[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    bool have_all = true;
    for (int q = 0; q < 6; ++q) {
        a.ix[q] = -1;
        for (int c = 0; c < sys->n_corr; ++c)
            if (sys->corr_a[c] == want[q][0] && sys->corr_b[c] == want[q][1]) a.ix[q] = c;
        have_all = have_all && a.ix[q] >= 0;
    }
    const bool planes = w || chi_frac || tr;
    if (planes && !have_all)
        return fail(PC_ERR_INVALID, "plane invariants need the correlators xx, yy, zz, xy, xz, yz");
    const size_t nv = size_t(a.n_corr) * size_t(a.n_k) * 2, np = size_t(K) * size_t(a.n_k);
    DevBuf<int32_t> d_slots;
    DevBuf<double> d_out;
    DevBuf<unsigned long long> d_max;
    PC_CK(d_slots.alloc(size_t(K)));
    PC_CK(d_out.alloc(4 * nv + (planes ? 3 * np : 0)));
    PC_CK(d_max.alloc(size_t(2 * K)));
    PC_CK(cudaMemcpyAsync(d_slots.p, slots, sizeof(int32_t) * size_t(K), cudaMemcpyHostToDevice, sys->stream));
    PC_CK(cudaMemsetAsync(d_max.p, 0, sizeof(unsigned long long) * size_t(2 * K), sys->stream));
    a.slots = d_slots.p;
    a.out_corr = d_out.p;
    a.out_corr2 = d_out.p + nv;
    a.out_var_inter = d_out.p + 2 * nv;
    a.out_var_intra = d_out.p + 3 * nv;
    if (planes) {
        a.w = d_out.p + 4 * nv;
        a.chi = a.w + np;
        a.tr = a.chi + np;
        a.max_bits = d_max.p;
    }
    pc::launch_ssf_merge(a, sys->stream);
    PC_LAUNCH_CK();
    sys->launches += planes ? 3 : 1;
    double* outs[7] = {static_corr, static_corr_2, var_inter, var_intra, w, chi_frac, tr};
    const double* src[7] = {a.out_corr, a.out_corr2, a.out_var_inter, a.out_var_intra, a.w, a.chi, a.tr};
    const size_t cnt[7] = {nv, nv, nv, nv, np, np, np};
    for (int i = 0; i < 7; ++i)
        if (outs[i] && src[i])
            PC_CK(cudaMemcpyAsync(outs[i], src[i], sizeof(double) * cnt[i], cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}

int pc_ssf_set_resolved(pc_system* sys, int resolved) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    sys->ssf_resolved = resolved != 0;
    sys->ssf_ready = false;  // accumulators change shape: configure again
    sys->drop_graphs();
    return PC_OK;
}

int pc_ssf_sample(pc_system* sys, const int32_t* slot_of_replica) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->ssf_ready) return fail(PC_ERR_STATE, "ssf not configured");
    for (int r = 0; r < sys->R; ++r) {
        const int s = slot_of_replica[r];
        if (s >= sys->n_slots) return fail(PC_ERR_INVALID, "slot index out of range");
        if (s >= 0 && sys->L_of_slot[size_t(s)] != sys->L[size_t(r)])
            return fail(PC_ERR_INVALID, "slot size differs from replica size");
    }
    PC_CK(cudaMemcpyAsync(sys->d_slot_of_rep.p, slot_of_replica, sizeof(int32_t) * size_t(sys->R),
                          cudaMemcpyHostToDevice, sys->stream));
    for (auto& g : sys->groups) {
        std::vector<int32_t> sel;
        for (int r : g.reps)
            if (slot_of_replica[r] >= 0) sel.push_back(r);
        g.n_sel = int(sel.size());
        if (!sel.empty())  // pageable source: the call returns once the data is staged
            PC_CK(cudaMemcpyAsync(g.d_sel_index.p, sel.data(), sizeof(int32_t) * sel.size(), cudaMemcpyHostToDevice,
                                  sys->stream));
    }
    pc::SsfOut o = ssf_out_base(sys);
    o.acc_sum = sys->d_ssf_sum.p;
    o.acc_sq = sys->d_ssf_sq.p;
    o.slot_of_rep = sys->d_slot_of_rep.p;
    rc = enqueue_ssf(sys, o, true);
    if (rc) return rc;
    for (int r = 0; r < sys->R; ++r)
        if (slot_of_replica[r] >= 0) sys->ssf_n[size_t(slot_of_replica[r])]++;
    return PC_OK;
}

int pc_ssf_read(pc_system* sys, int slot, double* sum, double* sq, uint64_t* n_samples) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->ssf_ready) return fail(PC_ERR_STATE, "ssf not configured");
    if (slot < 0 || slot >= sys->n_slots) return fail(PC_ERR_INVALID, "slot index out of range");
    const int L = sys->L_of_slot[size_t(slot)];
    const size_t n = size_t(sys->n_corr) * size_t(L) * L * L * 2 * (sys->ssf_resolved ? 256 : 1);
    PC_CK(cudaStreamSynchronize(sys->stream));
    if (sum)
        PC_CK(cudaMemcpy(sum, sys->d_ssf_sum.p + size_t(slot) * sys->slot_stride, sizeof(double) * n,
                         cudaMemcpyDeviceToHost));
    if (sq)
        PC_CK(cudaMemcpy(sq, sys->d_ssf_sq.p + size_t(slot) * sys->slot_stride, sizeof(double) * n,
                         cudaMemcpyDeviceToHost));
    if (n_samples) *n_samples = sys->ssf_n[size_t(slot)];
    return PC_OK;
}

int pc_ssf_clear(pc_system* sys, int slot) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->ssf_ready) return fail(PC_ERR_STATE, "ssf not configured");
    if (slot < 0 || slot >= sys->n_slots) return fail(PC_ERR_INVALID, "slot index out of range");
    PC_CK(cudaMemsetAsync(sys->d_ssf_sum.p + size_t(slot) * sys->slot_stride, 0, sizeof(double) * sys->slot_stride,
                          sys->stream));
    PC_CK(cudaMemsetAsync(sys->d_ssf_sq.p + size_t(slot) * sys->slot_stride, 0, sizeof(double) * sys->slot_stride,
                          sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    sys->ssf_n[size_t(slot)] = 0;
    return PC_OK;
}

namespace {
// S(q) of every replica into out_dev (see pc_ssf_forward), queued without
// waiting; with keep_amp the amplitudes B^a(K) stay in the groups' d_amp.
int ssf_forward_enqueue(pc_system* sys, void* out_dev, bool keep_amp) {
    if (!sys->ssf_ready) return fail(PC_ERR_STATE, "ssf not configured");
    if (sys->ssf_resolved) return fail(PC_ERR_UNSUPPORTED, "the differentiable S(q) is the contracted one");
    // out_dev is [R][n_corr][n_k][2] with replicas in index order; the kernel
    // indexes by position inside each size group, so offset per group.
    for (auto& g : sys->groups) {
        const size_t nk = size_t(g.L) * g.L * g.L;
        // groups must be replica-contiguous for the packed layout
        for (size_t i = 0; i < g.reps.size(); ++i)
            if (g.reps[i] != g.reps[0] + int(i)) return fail(PC_ERR_UNSUPPORTED, "ssf forward needs size-sorted replicas");
        pc::SsfOut o = ssf_out_base(sys);
        size_t off = 0;
        for (int r = 0; r < g.reps[0]; ++r) off += size_t(sys->n_corr) * size_t(sys->Nc(r)) * 2;
        o.val = static_cast<double*>(out_dev) + off;
        if (keep_amp) {
            if (g.d_amp.n != g.reps.size() * 3 * nk) PC_CK(g.d_amp.alloc(g.reps.size() * 3 * nk));
            o.amp = g.d_amp.p;
        }
        pc::SsfGeom geom{g.L, g.P, g.Q, int(g.reps.size()), g.d_rep_index.p};
        pc::launch_ssf_xy(geom, sys->d_spins.p, sys->d_reps.p, g.d_G.p, sys->stream);
        PC_LAUNCH_CK();
        pc::launch_ssf_z(geom, g.d_G.p, o, sys->stream);
        PC_LAUNCH_CK();
        sys->launches += 2;
    }
    return PC_OK;
}

// dLoss/dS_i into grad_S_dev (see pc_ssf_backward), queued without waiting;
// recompute: the forward amplitudes are formed again from the current spins
// (else the groups' d_amp holds them).
int ssf_backward_enqueue(pc_system* sys, const void* grad_out_dev, void* grad_S_dev, bool recompute) {
    if (!sys->ssf_ready) return fail(PC_ERR_STATE, "ssf not configured");
    if (sys->ssf_resolved) return fail(PC_ERR_UNSUPPORTED, "the differentiable S(q) is the contracted one");
    for (auto& g : sys->groups)
        for (size_t i = 0; i < g.reps.size(); ++i)
            if (g.reps[i] != g.reps[0] + int(i))
                return fail(PC_ERR_UNSUPPORTED, "ssf backward needs size-sorted replicas");
    PC_CK(cudaMemsetAsync(grad_S_dev, 0, sizeof(float4) * size_t(sys->N_tot), sys->stream));
    for (auto& g : sys->groups) {
        const size_t nk = size_t(g.L) * g.L * g.L;
        if (g.d_amp.n != g.reps.size() * 3 * nk) {
            PC_CK(g.d_amp.alloc(g.reps.size() * 3 * nk));
            recompute = true;
        }
        pc::SsfGeom geom{g.L, g.P, g.Q, int(g.reps.size()), g.d_rep_index.p};
        pc::SsfOut o = ssf_out_base(sys);
        o.amp = g.d_amp.p;
        if (recompute) {  // the forward amplitudes
            pc::launch_ssf_xy(geom, sys->d_spins.p, sys->d_reps.p, g.d_G.p, sys->stream);
            PC_LAUNCH_CK();
            pc::launch_ssf_z(geom, g.d_G.p, o, sys->stream);
            PC_LAUNCH_CK();
            sys->launches += 2;
        }
        size_t off = 0;
        for (int r = 0; r < g.reps[0]; ++r) off += size_t(sys->n_corr) * size_t(sys->Nc(r)) * 2;
        const double* dval = static_cast<const double*>(grad_out_dev) + off;
        pc::launch_ssf_adjoint(geom, o, dval, g.d_amp.p, g.d_G.p, static_cast<float4*>(grad_S_dev), sys->d_reps.p,
                               sys->stream);
        PC_LAUNCH_CK();
        sys->launches += 2;
    }
    return PC_OK;
}
}  // namespace

int pc_ssf_forward(pc_system* sys, void* out_dev) {
    int rc = check_sys(sys);
    if (rc) return rc;
    rc = ssf_forward_enqueue(sys, out_dev, false);
    if (rc) return rc;
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}

int pc_ssf_backward(pc_system* sys, const void* grad_out_dev, void* grad_S_dev) {
    int rc = check_sys(sys);
    if (rc) return rc;
    rc = ssf_backward_enqueue(sys, grad_out_dev, grad_S_dev, true);
    sys->amp_token = 0;  // the kept amplitudes were overwritten
    if (rc) return rc;
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}

int pc_ssf_forward_keep(pc_system* sys, void* out_dev, uint64_t* token) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!token) return fail(PC_ERR_INVALID, "pc_ssf_forward_keep: null token");
    *token = 0;
    sys->amp_token = 0;
    rc = ssf_forward_enqueue(sys, out_dev, true);
    if (rc) return rc;
    sys->amp_token = ++sys->amp_serial;
    *token = sys->amp_token;
    return PC_OK;
}

int pc_ssf_backward_kept(pc_system* sys, uint64_t token, const void* grad_out_dev, void* grad_S_dev) {
    int rc = check_sys(sys);
    if (rc) return rc;
    const bool kept = token != 0 && token == sys->amp_token;
    if (!kept) sys->amp_token = 0;
    return ssf_backward_enqueue(sys, grad_out_dev, grad_S_dev, !kept);
}

int pc_ssf_current(pc_system* sys, int replica, double* out) {
    int rc = check_sys(sys);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    if (!sys->ssf_ready) return fail(PC_ERR_STATE, "ssf not configured");
    const size_t n = size_t(sys->n_corr) * size_t(sys->Nc(replica)) * 2 * (sys->ssf_resolved ? 256 : 1);
    DevBuf<double> val;
    PC_CK(val.alloc(n));
    for (auto& g : sys->groups) {
        if (g.L != sys->L[size_t(replica)]) continue;
        DevBuf<int32_t> idx;
        PC_CK(idx.alloc(1));
        PC_CK(cudaMemcpy(idx.p, &replica, sizeof(int32_t), cudaMemcpyHostToDevice));
        pc::SsfGeom geom{g.L, g.P, g.Q, 1, idx.p, sys->ssf_resolved ? 1 : 0};
        pc::SsfOut o = ssf_out_base(sys);
        o.val = val.p;
        pc::launch_ssf_xy(geom, sys->d_spins.p, sys->d_reps.p, g.d_G.p, sys->stream);
        PC_LAUNCH_CK();
        pc::launch_ssf_z(geom, g.d_G.p, o, sys->stream);
        PC_LAUNCH_CK();
        sys->launches += 2;
        PC_CK(cudaStreamSynchronize(sys->stream));
        idx.release();
    }
    PC_CK(cudaMemcpy(out, val.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    val.release();
    return PC_OK;
}

int pc_spin_ft(pc_system* sys, int replica, double* out) {
    int rc = check_sys(sys);
    if (rc) return rc;
    rc = check_rep(sys, replica);
    if (rc) return rc;
    if (!out) return fail(PC_ERR_INVALID, "null output");
    rc = ensure_groups(sys);
    if (rc) return rc;
    const int L = sys->L[size_t(replica)];
    SsfGroup* grp = nullptr;
    for (auto& g : sys->groups)
        if (g.L == L) grp = &g;
    if (!grp || !pc::ssf_resolved_supported(grp->P, grp->Q))
        return fail(PC_ERR_UNSUPPORTED, "the per-sublattice transform needs L to factor into two parts <= 8");
    DevBuf<int32_t> idx;
    PC_CK(idx.alloc(1));
    PC_CK(cudaMemcpy(idx.p, &replica, sizeof(int32_t), cudaMemcpyHostToDevice));
    pc::SsfGeom geom{grp->L, grp->P, grp->Q, 1, idx.p, 1};
    pc::launch_ssf_xy(geom, sys->d_spins.p, sys->d_reps.p, grp->d_G.p, sys->stream);
    PC_LAUNCH_CK();
    pc::launch_ssf_zdft_res(geom, grp->d_G.p, sys->stream);
    PC_LAUNCH_CK();
    sys->launches += 2;
    const size_t L3 = size_t(L) * L * L;
    std::vector<float2> A(48 * L3);
    PC_CK(cudaMemcpyAsync(A.data(), grp->d_G.p, sizeof(float2) * A.size(), cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    // A[plane = 16 c + sl][Kz][Ky][Kx] -> out[c][sl][k = (Kx L + Ky) L + Kz][re, im]
    for (size_t pl = 0; pl < 48; ++pl)
        for (int kz = 0; kz < L; ++kz)
            for (int ky = 0; ky < L; ++ky)
                for (int kx = 0; kx < L; ++kx) {
                    const float2 v = A[pl * L3 + (size_t(kz) * L + ky) * L + kx];
                    double* o = out + (pl * L3 + (size_t(kx) * L + ky) * L + kz) * 2;
                    o[0] = v.x;
                    o[1] = v.y;
                }
    return PC_OK;
}

// ------------------------------------------------------------- tempering
int pc_pt_configure(pc_system* sys, const double* T) {
    int rc = check_sys(sys);
    if (rc) return rc;
    std::map<int, std::vector<int>> by_L;
    for (int r = 0; r < sys->R; ++r) {
        if (!(T[r] > 0)) return fail(PC_ERR_INVALID, "temperatures must be positive");
        by_L[sys->L[size_t(r)]].push_back(r);
    }
    std::vector<int32_t> rep_of_slot, slot_of_rep(size_t(sys->R));
    sys->ladder_begin.clear();
    sys->T_slot.clear();
    for (auto& kv : by_L) {
        auto reps = kv.second;
        std::stable_sort(reps.begin(), reps.end(), [&](int a, int b) { return T[a] > T[b]; });
        sys->ladder_begin.push_back(int32_t(rep_of_slot.size()));
        for (int r : reps) {
            slot_of_rep[size_t(r)] = int32_t(rep_of_slot.size());
            rep_of_slot.push_back(r);
            sys->T_slot.push_back(T[r]);
        }
    }
    sys->ladder_begin.push_back(int32_t(rep_of_slot.size()));
    sys->n_ladders = int(by_L.size());
    const size_t ns = rep_of_slot.size();
    PC_CK(sys->d_ladder_begin.alloc(sys->ladder_begin.size()));
    PC_CK(cudaMemcpy(sys->d_ladder_begin.p, sys->ladder_begin.data(), sizeof(int32_t) * sys->ladder_begin.size(),
                     cudaMemcpyHostToDevice));
    PC_CK(sys->d_rep_of_slot.alloc(ns));
    PC_CK(cudaMemcpy(sys->d_rep_of_slot.p, rep_of_slot.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice));
    PC_CK(sys->d_pt_slot_of_rep.alloc(ns));
    PC_CK(cudaMemcpy(sys->d_pt_slot_of_rep.p, slot_of_rep.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice));
    PC_CK(sys->d_T_slot.alloc(ns));
    PC_CK(cudaMemcpy(sys->d_T_slot.p, sys->T_slot.data(), sizeof(double) * ns, cudaMemcpyHostToDevice));
    PC_CK(cudaMemcpy(sys->d_T.p, T, sizeof(double) * ns, cudaMemcpyHostToDevice));
    PC_CK(sys->d_E_sum.alloc(ns));
    PC_CK(sys->d_E2_sum.alloc(ns));
    PC_CK(sys->d_n_e.alloc(ns));
    PC_CK(sys->d_att.alloc(ns));
    PC_CK(sys->d_accn.alloc(ns));
    PC_CK(cudaMemset(sys->d_E_sum.p, 0, sizeof(double) * ns));
    PC_CK(cudaMemset(sys->d_E2_sum.p, 0, sizeof(double) * ns));
    PC_CK(cudaMemset(sys->d_n_e.p, 0, sizeof(unsigned long long) * ns));
    PC_CK(cudaMemset(sys->d_att.p, 0, sizeof(unsigned long long) * ns));
    PC_CK(cudaMemset(sys->d_accn.p, 0, sizeof(unsigned long long) * ns));
    PC_CK(sys->d_round.alloc(1));
    PC_CK(cudaMemset(sys->d_round.p, 0, sizeof(uint64_t)));
    sys->pt_sweeps_done = 0;
    sys->pt_ready = true;
    sys->drop_graphs();
    return PC_OK;
}

namespace {
pc::PtArgs pt_args(pc_system* s) {
    pc::PtArgs a;
    a.n_ladders = s->n_ladders;
    a.ladder_begin = s->d_ladder_begin.p;
    a.T_slot = s->d_T_slot.p;
    a.rep_of_slot = s->d_rep_of_slot.p;
    a.slot_of_rep = s->d_pt_slot_of_rep.p;
    a.T_rep = s->d_T.p;
    a.Tq = s->d_Tq.p;
    a.inv_T_ref = float(1.0 / s->T_ref);
    a.e_rep = s->d_e.p;
    a.reps = s->d_reps.p;
    a.E_sum = s->d_E_sum.p;
    a.E2_sum = s->d_E2_sum.p;
    a.n_e = s->d_n_e.p;
    a.attempts = s->d_att.p;
    a.accepts = s->d_accn.p;
    a.round = s->d_round.p;
    a.seed = s->seed;
    a.n_slots = int(s->T_slot.size());
    return a;
}

int enqueue_pt_round(pc_system* s, int n_sweep, int ssf_every, uint64_t sweep_phase) {
    for (int i = 0; i < n_sweep; ++i) {
        int rc = enqueue_sweep(s, uint64_t(i), 1, false);
        if (rc) return rc;
        if (ssf_every > 0 && (sweep_phase + uint64_t(i) + 1) % uint64_t(ssf_every) == 0) {
            pc::SsfOut o = ssf_out_base(s);
            o.acc_sum = s->d_ssf_sum.p;
            o.acc_sq = s->d_ssf_sq.p;
            o.slot_of_rep = s->d_pt_slot_of_rep.p;
            rc = enqueue_ssf(s, o, false);
            if (rc) return rc;
        }
    }
    pc::launch_advance_counter(s->d_sweep.p, uint64_t(n_sweep), s->stream);
    PC_LAUNCH_CK();
    s->launches++;
    int rc = enqueue_energy(s);
    if (rc) return rc;
    pc::launch_pt_exchange(pt_args(s), s->stream);
    PC_LAUNCH_CK();
    s->launches++;
    return PC_OK;
}

// Why the rounds of this system cannot run in the persistent kernel (nullptr:
// they can): it covers the structured couplings with standard Metropolis
// moves, rotation overrelaxation, the fused or reference-order schedule and
// the per-site neighbour loads (not the staged rows).
const char* pt_persistent_unsupported(pc_system* s) {
    if (!s->structured) return "the persistent tempering kernel needs the pyrochlore couplings";
    if (s->update != 0) return "the persistent tempering kernel runs standard Metropolis moves";
    if (s->or_mode != 0) return "the persistent tempering kernel runs rotation overrelaxation";
    if (s->schedule > 1) return "the persistent tempering kernel runs the fused or reference-order schedule";
    if (use_staged(s)) return "the persistent tempering kernel does not run the staged row tiles";
    if (s->threads < 32 || s->threads > 256 || s->threads % 32) return "the persistent tempering kernel needs 32..256 threads";
    return nullptr;
}

// One persistent launch: n_rounds rounds of n_sweep sweeps, each followed by
// the energies and the exchange when `exchange`.
int launch_persistent(pc_system* s, int n_rounds, int n_sweep, int exchange) {
    const int fused = s->schedule == 1 ? 1 : 0;
    const std::array<int, 3> key = {s->iso_kind, fused, s->threads};
    auto it = s->persist_cap.find(key);
    if (it == s->persist_cap.end())
        it = s->persist_cap.emplace(key, pc::pt_persistent_capacity(s->iso_kind, fused, s->threads)).first;
    if (it->second <= 0) return fail(PC_ERR_UNSUPPORTED, "no cooperative launch of the persistent kernel fits");
    // as few blocks as give every block the same number of tiles of the largest
    // colour class: each pass ends at a barrier, so the block with the most
    // tiles sets its length
    int most = 1;
    for (int c = 0; c < s->n_colours; ++c) most = std::max(most, s->n_colour_tiles[size_t(c)]);
    const int per_block = (most + it->second - 1) / it->second;
    const int grid = std::max(1, (most + per_block - 1) / per_block);
    pc::PersistArgs p;
    std::memset(&p, 0, sizeof(p));
    p.pass = pass_args(s, 0, 0, 0);
    for (int c = 0; c < s->n_colours; ++c) {
        p.colour_tiles[c] = s->d_colour_tiles[size_t(c)].p;
        p.n_colour_tiles[c] = s->n_colour_tiles[size_t(c)];
    }
    p.n_colours = s->n_colours;
    p.fused = fused;
    p.n_rounds = n_rounds;
    p.n_sweep = n_sweep;
    p.exchange = exchange;
    p.sweep = s->d_sweep.p;
    p.c_tiles = s->d_cell_tiles.p;
    p.n_c_tiles = s->n_cell_tiles;
    p.uniform = s->iso_uniform ? 1 : 0;
    p.partial = s->d_cell_partial.p;
    p.c_begin = s->d_cell_begin.p;
    p.c_end = s->d_cell_end.p;
    p.e = s->d_e.p;
    p.mag = s->d_mag.p;
    p.R = s->R;
    p.pt = pt_args(s);
    p.bar = s->d_bar.p;
    p.max_polls = s->barrier_polls;
    PC_CK(cudaMemsetAsync(s->d_bar.p, 0, pc::kBarrierWords * sizeof(unsigned int), s->stream));
    const int e = pc::launch_pt_persistent(p, s->iso_kind, grid, s->threads, s->stream);
    if (e != 0) return fail(PC_ERR_CUDA, std::string("persistent launch: ") + cudaGetErrorString(cudaError_t(e)));
    s->launches++;
    return PC_OK;
}

// pc_pt_run on the persistent kernel. Without S(q) samples, all rounds are one
// launch. With samples, a round is split at the sweeps after which S(q) is
// sampled (the S(q) kernels run between the launches), and its energies and
// exchange come last, after a sample that follows the round's last sweep, as
// in the per-pass schedule.
int run_pt_persistent(pc_system* s, int n_rounds, int n_sweep, int ssf_every) {
    if (!s->d_bar.p) PC_CK(s->d_bar.alloc(pc::kBarrierWords));
    PC_CK(cudaMemsetAsync(s->d_err.p, 0, sizeof(int), s->stream));
    if (ssf_every <= 0) {
        int rc = n_rounds > 0 ? launch_persistent(s, n_rounds, n_sweep, 1) : PC_OK;
        if (rc) return rc;
        s->pt_sweeps_done += uint64_t(n_rounds) * uint64_t(n_sweep);
        s->host_sweep += uint64_t(n_rounds) * uint64_t(n_sweep);
        return device_error(s);
    }
    for (int round = 0; round < n_rounds; ++round) {
        const uint64_t phase = s->pt_sweeps_done % uint64_t(ssf_every);
        int start = 0;
        for (int i = 0; i < n_sweep; ++i) {
            if ((phase + uint64_t(i) + 1) % uint64_t(ssf_every) != 0) continue;
            const bool last = i + 1 == n_sweep;
            int rc = launch_persistent(s, 1, i + 1 - start, 0);
            if (rc) return rc;
            pc::SsfOut o = ssf_out_base(s);
            o.acc_sum = s->d_ssf_sum.p;
            o.acc_sq = s->d_ssf_sq.p;
            o.slot_of_rep = s->d_pt_slot_of_rep.p;
            rc = enqueue_ssf(s, o, false);
            if (rc) return rc;
            for (auto& n : s->ssf_n) n++;
            start = i + 1;
            if (last) break;
        }
        int rc = launch_persistent(s, 1, n_sweep - start, 1);
        if (rc) return rc;
        s->pt_sweeps_done += uint64_t(n_sweep);
        s->host_sweep += uint64_t(n_sweep);
    }
    return device_error(s);
}
}  // namespace

int pc_pt_run(pc_system* sys, int n_rounds, int n_sweep, int ssf_every) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->pt_ready) return fail(PC_ERR_STATE, "tempering not configured");
    if (n_rounds < 0 || n_sweep < 1 || ssf_every < 0) return fail(PC_ERR_INVALID, "bad tempering schedule");
    if (ssf_every > 0) {
        if (!sys->ssf_ready || sys->n_slots != int(sys->T_slot.size()))
            return fail(PC_ERR_STATE, "tempering SSF needs pc_ssf_configure with one slot per replica");
        for (size_t sl = 0; sl < sys->T_slot.size(); ++sl) {
            int32_t r = -1;
            PC_CK(cudaMemcpy(&r, sys->d_rep_of_slot.p + sl, sizeof(int32_t), cudaMemcpyDeviceToHost));
            if (sys->L_of_slot[sl] != sys->L[size_t(r)])
                return fail(PC_ERR_INVALID, "tempering SSF slot sizes must follow the ladders (ascending L)");
        }
    }
    PC_CK(cudaMemsetAsync(sys->d_acc.p, 0, sizeof(unsigned long long) * size_t(sys->R), sys->stream));
    rc = refresh_tq(sys);
    if (rc) return rc;
    if (sys->pt_persistent) {
        if (const char* why = pt_persistent_unsupported(sys)) return fail(PC_ERR_UNSUPPORTED, why);
        return run_pt_persistent(sys, n_rounds, n_sweep, ssf_every);
    }
    const uint64_t period = ssf_every > 0 ? uint64_t(ssf_every) : 1;
    for (int round = 0; round < n_rounds; ++round) {
        const uint64_t phase = sys->pt_sweeps_done % period;
        const auto key = std::make_pair(n_sweep, int(ssf_every > 0 ? phase : 0) + 100000 * ssf_every);
        auto it = sys->pt_graphs.find(key);
        if (it == sys->pt_graphs.end()) {
            const uint64_t before = sys->launches;
            PC_CK(cudaStreamBeginCapture(sys->stream, cudaStreamCaptureModeThreadLocal));
            rc = enqueue_pt_round(sys, n_sweep, ssf_every, phase);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(sys->stream, &g);
            if (rc) return rc;
            if (e != cudaSuccess) return fail(PC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            cudaGraphExec_t x = nullptr;
            PC_CK(cudaGraphInstantiate(&x, g, 0));
            cudaGraphDestroy(g);
            const int nodes = int(sys->launches - before);
            sys->launches = before;
            it = sys->pt_graphs.insert({key, {x, nodes}}).first;
        }
        PC_CK(cudaGraphLaunch(it->second.first, sys->stream));
        sys->launches += uint64_t(it->second.second);
        // host-side SSF sample counts (every slot samples together)
        if (ssf_every > 0)
            for (int i = 0; i < n_sweep; ++i)
                if ((phase + uint64_t(i) + 1) % uint64_t(ssf_every) == 0)
                    for (auto& n : sys->ssf_n) n++;
        sys->pt_sweeps_done += uint64_t(n_sweep);
        sys->host_sweep += uint64_t(n_sweep);
    }
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}

int pc_pt_reset_stats(pc_system* sys) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->pt_ready) return fail(PC_ERR_STATE, "tempering not configured");
    const size_t ns = sys->T_slot.size();
    PC_CK(cudaMemsetAsync(sys->d_E_sum.p, 0, sizeof(double) * ns, sys->stream));
    PC_CK(cudaMemsetAsync(sys->d_E2_sum.p, 0, sizeof(double) * ns, sys->stream));
    PC_CK(cudaMemsetAsync(sys->d_n_e.p, 0, sizeof(unsigned long long) * ns, sys->stream));
    PC_CK(cudaMemsetAsync(sys->d_att.p, 0, sizeof(unsigned long long) * ns, sys->stream));
    PC_CK(cudaMemsetAsync(sys->d_accn.p, 0, sizeof(unsigned long long) * ns, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    return PC_OK;
}

int pc_pt_read_energy(pc_system* sys, double* T, double* E, double* E2, uint64_t* n) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->pt_ready) return fail(PC_ERR_STATE, "tempering not configured");
    const size_t ns = sys->T_slot.size();
    PC_CK(cudaStreamSynchronize(sys->stream));
    if (T) std::memcpy(T, sys->T_slot.data(), sizeof(double) * ns);
    if (E) PC_CK(cudaMemcpy(E, sys->d_E_sum.p, sizeof(double) * ns, cudaMemcpyDeviceToHost));
    if (E2) PC_CK(cudaMemcpy(E2, sys->d_E2_sum.p, sizeof(double) * ns, cudaMemcpyDeviceToHost));
    if (n) PC_CK(cudaMemcpy(n, sys->d_n_e.p, sizeof(uint64_t) * ns, cudaMemcpyDeviceToHost));
    return PC_OK;
}
int pc_pt_read_exchange(pc_system* sys, uint64_t* attempts, uint64_t* accepts) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->pt_ready) return fail(PC_ERR_STATE, "tempering not configured");
    const size_t ns = sys->T_slot.size();
    PC_CK(cudaStreamSynchronize(sys->stream));
    PC_CK(cudaMemcpy(attempts, sys->d_att.p, sizeof(uint64_t) * ns, cudaMemcpyDeviceToHost));
    PC_CK(cudaMemcpy(accepts, sys->d_accn.p, sizeof(uint64_t) * ns, cudaMemcpyDeviceToHost));
    return PC_OK;
}
int pc_pt_slots(pc_system* sys, int32_t* slot_of_replica) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->pt_ready) return fail(PC_ERR_STATE, "tempering not configured");
    PC_CK(cudaStreamSynchronize(sys->stream));
    PC_CK(cudaMemcpy(slot_of_replica, sys->d_pt_slot_of_rep.p, sizeof(int32_t) * size_t(sys->R), cudaMemcpyDeviceToHost));
    return PC_OK;
}

// -------------------------------------------------------------- gradients
namespace {
int energy_grad_of(pc_system* sys, const float4* spins, const double* g, double* e_per_cell, void* grad_S_dev,
                   double* grad_J, double* grad_B);
int enqueue_energy_grad(pc_system* sys, const float4* spins, const double* g_dev, void* grad_S_dev, bool want_J,
                        int* width_out);
}

int pc_energy_grad(pc_system* sys, const double* g, double* e_per_cell, void* grad_S_dev, double* grad_J,
                   double* grad_B) {
    int rc = check_sys(sys);
    if (rc) return rc;
    return energy_grad_of(sys, sys->d_spins.p, g, e_per_cell, grad_S_dev, grad_J, grad_B);
}

int pc_energy_device(pc_system* sys, double* e_dev) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!e_dev || reinterpret_cast<uintptr_t>(e_dev) % 8 != 0)
        return fail(PC_ERR_INVALID, "pc_energy_device: null or misaligned output");
    rc = enqueue_energy(sys);
    if (rc) return rc;
    PC_CK(cudaMemcpyAsync(e_dev, sys->d_e.p, sizeof(double) * size_t(sys->R), cudaMemcpyDeviceToDevice, sys->stream));
    return PC_OK;
}

int pc_energy_groups_device(pc_system* sys, double* e_dev, double* out_dev) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!sys->structured || sys->iso_kind != 1 || !sys->iso_uniform)
        return fail(PC_ERR_UNSUPPORTED, "pc_energy_groups_device needs isotropic couplings, every group nonzero and "
                                        "the same on all sublattices");
    if (!e_dev || !out_dev || reinterpret_cast<uintptr_t>(e_dev) % 8 != 0 ||
        reinterpret_cast<uintptr_t>(out_dev) % 8 != 0)
        return fail(PC_ERR_INVALID, "pc_energy_groups_device: null or misaligned output");
    rc = enqueue_energy(sys, true);
    if (rc) return rc;
    const size_t R = size_t(sys->R), row = size_t(pc::kGroups + 3) * sizeof(double);
    PC_CK(cudaMemcpyAsync(e_dev, sys->d_e.p, sizeof(double) * R, cudaMemcpyDeviceToDevice, sys->stream));
    PC_CK(cudaMemcpy2DAsync(out_dev, row, sys->d_group_out.p, pc::kGroups * sizeof(double),
                            pc::kGroups * sizeof(double), R, cudaMemcpyDeviceToDevice, sys->stream));
    PC_CK(cudaMemcpy2DAsync(out_dev + pc::kGroups, row, sys->d_mag.p, 3 * sizeof(double), 3 * sizeof(double), R,
                            cudaMemcpyDeviceToDevice, sys->stream));
    return PC_OK;
}

int pc_energy_grad_device(pc_system* sys, const double* g_dev, void* grad_S_dev, double* sums_dev, int couplings) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if ((g_dev && reinterpret_cast<uintptr_t>(g_dev) % 8 != 0) ||
        (grad_S_dev && reinterpret_cast<uintptr_t>(grad_S_dev) % 16 != 0) ||
        (sums_dev && reinterpret_cast<uintptr_t>(sums_dev) % 8 != 0))
        return fail(PC_ERR_INVALID, "pc_energy_grad_device: misaligned pointer");
    const size_t R = size_t(sys->R);
    if (!g_dev) {  // g = 1 for every replica
        if (sys->d_grad_ones.n != R) {
            PC_CK(sys->d_grad_ones.alloc(R));
            const std::vector<double> ones(R, 1.0);
            PC_CK(cudaMemcpy(sys->d_grad_ones.p, ones.data(), sizeof(double) * R, cudaMemcpyHostToDevice));
        }
        g_dev = sys->d_grad_ones.p;
    }
    int width = 0;
    rc = enqueue_energy_grad(sys, sys->d_spins.p, g_dev, grad_S_dev, couplings != 0, &width);
    if (rc) return rc;
    if (sums_dev) {
        const size_t row = size_t(4 + 9 * int(sys->specs.size()));
        const size_t cols = couplings ? row : 4;
        PC_CK(cudaMemcpy2DAsync(sums_dev, row * sizeof(double), sys->d_grad_out.p, size_t(width) * sizeof(double),
                                cols * sizeof(double), R, cudaMemcpyDeviceToDevice, sys->stream));
    }
    return PC_OK;
}

int pc_energy_grad_field(pc_system* sys, const void* field_dev, const double* g, double* e_per_cell,
                         void* grad_S_dev, double* grad_J, double* grad_B) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!field_dev) return fail(PC_ERR_INVALID, "pc_energy_grad_field: null field");
    if (reinterpret_cast<uintptr_t>(field_dev) % 16 != 0)
        return fail(PC_ERR_INVALID, "pc_energy_grad_field: field is not 16-byte aligned (float4)");
    if (grad_S_dev == field_dev) return fail(PC_ERR_INVALID, "pc_energy_grad_field: output aliases the field");
    return energy_grad_of(sys, static_cast<const float4*>(field_dev), g, e_per_cell, grad_S_dev, grad_J, grad_B);
}

}  // extern "C"

namespace {
// Queues the gradient kernels for the upstream g_dev (device, one double per
// replica) on the system's stream; the per-replica sums land in d_grad_out,
// *width doubles a replica: [sum of the owned bond energies - S.B, sum S (3),
// the 9 * n_spec coupling products when formed].
int enqueue_energy_grad(pc_system* sys, const float4* spins, const double* g_dev, void* grad_S_dev, bool want_J,
                        int* width_out) {
    const int ns = int(sys->specs.size());
    // the structured kernel forms the coupling products only when they are asked for
    const bool structured = sys->grad_struct && sys->threads <= 256;
    const int width = (structured && !want_J) ? 4 : 4 + 9 * ns;
    if (sys->d_grad_out.n < size_t(sys->R) * size_t(4 + 9 * ns))  // the widest form, kept across calls
        PC_CK(sys->d_grad_out.alloc(size_t(sys->R) * size_t(4 + 9 * ns)));
    DevBuf<double>& d_out = sys->d_grad_out;
    if (structured) {
        pc::GradStructArgs a;
        a.spins = spins;
        a.reps = sys->d_reps.p;
        a.tiles = sys->d_all_tiles.p;
        a.items = sys->d_grad_items.p;
        a.n_items = sys->n_grad_items;
        a.width = width;
        for (int i = 0; i < 3; ++i) a.B[i] = float(sys->B[i]);
        a.g = g_dev;
        a.grad_S = static_cast<float4*>(grad_S_dev);
        a.partial = sys->d_grad_partial.p;
        a.mats = sys->mats;
        std::memcpy(a.spec_mask, sys->spec_mask, sizeof(a.spec_mask));
        pc::launch_energy_grad_struct(a, want_J, sys->threads, sys->stream);
        PC_LAUNCH_CK();
        pc::launch_grad_finalize(sys->d_grad_partial.p, width, sys->d_item_begin.p, sys->d_item_end.p, sys->R,
                                 d_out.p, sys->stream);
        PC_LAUNCH_CK();
    } else {
        pc::GradArgs a;
        a.spins = spins;
        a.reps = sys->d_reps.p;
        a.tables = sys->d_tab_full.p;
        a.tiles = sys->d_all_tiles.p;
        a.n_tiles = sys->n_all_tiles;
        a.n_spec = ns;
        for (int i = 0; i < 3; ++i) a.B[i] = float(sys->B[i]);
        a.g = g_dev;
        a.grad_S = static_cast<float4*>(grad_S_dev);
        a.partial = sys->d_partial.p;
        pc::launch_energy_grad_partials(a, sys->threads, sys->stream);
        PC_LAUNCH_CK();
        pc::launch_grad_finalize(sys->d_partial.p, width, sys->d_tile_begin.p, sys->d_tile_end.p, sys->R, d_out.p,
                                 sys->stream);
        PC_LAUNCH_CK();
    }
    sys->launches += 2;
    *width_out = width;
    return PC_OK;
}

int energy_grad_of(pc_system* sys, const float4* spins, const double* g, double* e_per_cell, void* grad_S_dev,
                   double* grad_J, double* grad_B) {
    const int ns = int(sys->specs.size());
    if (sys->d_grad_g.n != size_t(sys->R)) PC_CK(sys->d_grad_g.alloc(size_t(sys->R)));
    const size_t R = size_t(sys->R);
    PC_CK(sys->stage(sizeof(double) * R * size_t(1 + 4 + 9 * ns)));
    double* st_g = static_cast<double*>(sys->h_stage);
    double* st_out = st_g + R;
    for (size_t r = 0; r < R; ++r) st_g[r] = g ? g[r] : 1.0;
    PC_CK(cudaMemcpyAsync(sys->d_grad_g.p, st_g, sizeof(double) * R, cudaMemcpyHostToDevice, sys->stream));
    int width = 0;
    const int rc = enqueue_energy_grad(sys, spins, sys->d_grad_g.p, grad_S_dev, grad_J != nullptr, &width);
    if (rc) return rc;
    PC_CK(cudaMemcpyAsync(st_out, sys->d_grad_out.p, sizeof(double) * R * size_t(width), cudaMemcpyDeviceToHost,
                          sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    for (int r = 0; r < sys->R; ++r) {
        const double* o = st_out + size_t(r) * size_t(width);
        const double nc = double(sys->Nc(r));
        const double gr = g ? g[r] : 1.0;
        if (e_per_cell) e_per_cell[r] = o[0] / nc;
        if (grad_B)
            for (int a3 = 0; a3 < 3; ++a3) grad_B[3 * r + a3] = -gr * o[1 + a3] / nc;
        if (grad_J)
            for (int k = 0; k < 9 * ns; ++k) grad_J[size_t(r) * 9 * size_t(ns) + size_t(k)] = gr * o[4 + k] / nc;
    }
    return PC_OK;
}
}  // namespace

extern "C" {

// ---------------------------------------------------------------- tuning
int pc_get_tile(pc_system* sys, int* threads, int* ctas_per_sm) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    *threads = sys->threads;
    *ctas_per_sm = sys->ctas_per_sm;
    return PC_OK;
}
int pc_set_tile(pc_system* sys, int threads, int ctas_per_sm) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (threads < 32 || threads > 512 || threads % 32 != 0) return fail(PC_ERR_INVALID, "threads must be 32..512, a multiple of 32");
    if (ctas_per_sm < 0 || ctas_per_sm > 32)
        return fail(PC_ERR_INVALID, "ctas_per_sm must be 0 (one CTA per tile) or 1..32");
    sys->threads = threads;
    sys->ctas_per_sm = ctas_per_sm;
    if (sys->ready) return build_tiles(sys);
    return PC_OK;
}

int pc_set_load_variant(pc_system* sys, int variant) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (variant < 0 || variant > 3) return fail(PC_ERR_INVALID, "load variant must be 0, 1, 2 or 3");
    sys->load_variant = variant;
    sys->drop_graphs();
    if (sys->ready) return build_tiles(sys);  // variant 3 uses row tiles
    return PC_OK;
}
int pc_get_load_variant(pc_system* sys, int* variant) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    *variant = sys->load_variant;
    return PC_OK;
}

int pc_autotune(pc_system* sys) {
    int rc = check_sys(sys);
    if (rc) return rc;
    const size_t bytes = sizeof(float4) * size_t(sys->N_tot);
    DevBuf<float4> saved;
    PC_CK(saved.alloc(size_t(sys->N_tot)));
    PC_CK(cudaMemcpyAsync(saved.p, sys->d_spins.p, bytes, cudaMemcpyDeviceToDevice, sys->stream));
    uint64_t sweep0 = 0;
    PC_CK(cudaMemcpyAsync(&sweep0, sys->d_sweep.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    // the timing runs sweep at T = 1; the temperatures (a tempering ladder's
    // current assignment included) are put back afterwards, like the spins
    std::vector<double> T_saved(size_t(sys->R));
    PC_CK(cudaMemcpy(T_saved.data(), sys->d_T.p, sizeof(double) * T_saved.size(), cudaMemcpyDeviceToHost));
    std::vector<double> T(size_t(sys->R), 1.0);
    PC_CK(cudaMemcpy(sys->d_T.p, T.data(), sizeof(double) * T.size(), cudaMemcpyHostToDevice));
    // candidates: neighbour-load variant x threads per CTA x resident CTAs per
    // SM (the structured kernels run at most 256 threads per CTA)
    // (ctas 0: one CTA per tile, the hardware balancing the waves)
    const int cand_threads[4] = {64, 128, 256, 512};
    const int cand_ctas[8] = {0, 2, 3, 4, 5, 6, 7, 8};
    int best_t = sys->threads, best_c = sys->ctas_per_sm, best_v = sys->load_variant;
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    PC_CK(cudaEventCreate(&e0));
    PC_CK(cudaEventCreate(&e1));
    const bool timing = sys->timing;
    sys->timing = false;
    sys->cluster_sweep = false;
    const int n_var = sys->structured ? 4 : 1;
    for (int vi = 0; vi < n_var; ++vi)
        for (int ti = 0; ti < 4; ++ti)
            for (int ci = 0; ci < 8; ++ci) {
                if (sys->structured && cand_threads[ti] > 256) continue;
                sys->load_variant = vi;
                sys->threads = cand_threads[ti];
                sys->ctas_per_sm = cand_ctas[ci];
                if (vi == 3 && (!use_staged(sys) || ci > 0)) continue;  // row tiles: one CTA per tile
                rc = build_tiles(sys);
                if (rc) return rc;
                rc = run_sweeps(sys, 2, 1);  // warm-up + graph instantiation
                if (rc) return rc;
                float ms = 1e30f;  // best of three repeats: robust against a noisy neighbour
                for (int rep = 0; rep < 3; ++rep) {
                    PC_CK(cudaEventRecord(e0, sys->stream));
                    rc = run_sweeps(sys, 4, 1);
                    if (rc) return rc;
                    PC_CK(cudaEventRecord(e1, sys->stream));
                    PC_CK(cudaEventSynchronize(e1));
                    float t = 0.f;
                    PC_CK(cudaEventElapsedTime(&t, e0, e1));
                    ms = std::min(ms, t);
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best_t = cand_threads[ti];
                    best_c = cand_ctas[ci];
                    best_v = vi;
                }
            }
    // cluster-resident sweeps (small lattices): one more candidate
    if (cluster_eligible(sys, 1)) {
        sys->cluster_sweep = true;
        rc = run_sweeps(sys, 2, 1);
        if (rc) return rc;
        float ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            PC_CK(cudaEventRecord(e0, sys->stream));
            rc = run_sweeps(sys, 4, 1);
            if (rc) return rc;
            PC_CK(cudaEventRecord(e1, sys->stream));
            PC_CK(cudaEventSynchronize(e1));
            float t = 0.f;
            PC_CK(cudaEventElapsedTime(&t, e0, e1));
            ms = std::min(ms, t);
        }
        sys->cluster_sweep = ms < best_ms;
    }
    sys->threads = best_t;
    sys->ctas_per_sm = best_c;
    sys->load_variant = best_v;
    rc = build_tiles(sys);
    if (rc) return rc;
    // launch overlap of the colour passes, off and on, on the chosen tile (it
    // pays where passes are short: small lattices); the same moves either way
    if (!sys->cluster_sweep) {
        float ms_pdl[2] = {1e30f, 1e30f};
        for (int on = 0; on < 2; ++on) {
            sys->pdl = on != 0;
            sys->drop_graphs();
            rc = run_sweeps(sys, 2, 1);
            if (rc) return rc;
            for (int rep = 0; rep < 3; ++rep) {
                PC_CK(cudaEventRecord(e0, sys->stream));
                rc = run_sweeps(sys, 4, 1);
                if (rc) return rc;
                PC_CK(cudaEventRecord(e1, sys->stream));
                PC_CK(cudaEventSynchronize(e1));
                float t = 0.f;
                PC_CK(cudaEventElapsedTime(&t, e0, e1));
                ms_pdl[on] = std::min(ms_pdl[on], t);
            }
        }
        sys->pdl = ms_pdl[1] < ms_pdl[0];
        sys->drop_graphs();
    }
    sys->timing = timing;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PC_CK(cudaMemcpyAsync(sys->d_spins.p, saved.p, bytes, cudaMemcpyDeviceToDevice, sys->stream));
    PC_CK(cudaMemcpyAsync(sys->d_sweep.p, &sweep0, sizeof(uint64_t), cudaMemcpyHostToDevice, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    PC_CK(cudaMemcpy(sys->d_T.p, T_saved.data(), sizeof(double) * T_saved.size(), cudaMemcpyHostToDevice));
    sys->host_sweep = sweep0;
    saved.release();
    return PC_OK;
}

// --------------------------------------------------------------- bench API
namespace {
// The host-buffer step of pc_step_host (float4 spins, packed = false) and
// pc_step_host3 (packed (x, y, z) spins, unpacked and packed on the device in
// a staging buffer).
int step_host(pc_system* sys, const float* S_in, float* S_out, bool packed, double T, int n_sweep, int ssf_every,
              int ssf_slot, double* e_out, uint64_t* accepted) {
    int rc = check_sys(sys);
    if (rc) return rc;
    if (!(T > 0)) return fail(PC_ERR_INVALID, "temperature must be positive");
    if (n_sweep < 0 || ssf_every < 0) return fail(PC_ERR_INVALID, "bad sweep counts");
    const bool do_ssf = ssf_slot >= 0 && ssf_every > 0;
    if (do_ssf && (!sys->ssf_ready || ssf_slot >= sys->n_slots || sys->L_of_slot[size_t(ssf_slot)] != sys->L[0]))
        return fail(PC_ERR_STATE, "ssf slot not configured for replica 0");
    const int64_t n0 = sys->N(0);
    const size_t bytes = (packed ? 3 * sizeof(float) : sizeof(float4)) * size_t(n0);
    if (packed && sys->d_stage3.n < size_t(3 * n0)) PC_CK(sys->d_stage3.alloc(size_t(3 * n0)));
    void* dev_io = packed ? static_cast<void*>(sys->d_stage3.p) : static_cast<void*>(sys->d_spins.p);
    if (!sys->copy_stream) {
        PC_CK(cudaStreamCreateWithFlags(&sys->copy_stream, cudaStreamNonBlocking));
        PC_CK(cudaEventCreateWithFlags(&sys->ev_swept, cudaEventDisableTiming));
    }
    const size_t R = size_t(sys->R);
    PC_CK(sys->stage(sizeof(double) * R + 2 * sizeof(uint64_t) + sizeof(int)));
    double* st_T = static_cast<double*>(sys->h_stage);
    double* st_e = st_T + R;
    uint64_t* st_acc = reinterpret_cast<uint64_t*>(st_e + 1);
    int* st_flag = reinterpret_cast<int*>(st_acc + 1);
    PC_CK(cudaMemcpyAsync(dev_io, S_in, bytes, cudaMemcpyHostToDevice, sys->stream));
    if (packed) {
        pc::launch_spins_from_xyz(sys->d_spins.p, sys->d_stage3.p, n0, sys->stream);
        PC_LAUNCH_CK();
        sys->launches++;
    }
    for (size_t r = 0; r < R; ++r) st_T[r] = T;
    PC_CK(cudaMemcpyAsync(sys->d_T.p, st_T, sizeof(double) * R, cudaMemcpyHostToDevice, sys->stream));
    PC_CK(cudaMemsetAsync(sys->d_acc.p, 0, sizeof(unsigned long long) * size_t(sys->R), sys->stream));
    SsfGroup* grp = nullptr;
    if (do_ssf) {
        std::vector<int32_t> slots(size_t(sys->R), -1);
        slots[0] = ssf_slot;
        PC_CK(cudaMemcpyAsync(sys->d_slot_of_rep.p, slots.data(), sizeof(int32_t) * slots.size(), cudaMemcpyHostToDevice,
                              sys->stream));
        for (auto& g : sys->groups)
            if (g.L == sys->L[0]) grp = &g;
    }
    int done = 0;
    bool copying = false;
    // once the result copy is enqueued, every return (error paths included)
    // waits for it: the caller may reuse or free S_out as soon as we return
    struct CopyWait {
        const bool& active;
        cudaStream_t s;
        ~CopyWait() {
            if (active) cudaStreamSynchronize(s);
        }
    } copy_wait{copying, sys->copy_stream};
    while (done < n_sweep || !copying) {
        const int chunk = do_ssf ? std::min(ssf_every, n_sweep - done) : n_sweep - done;
        if (chunk > 0) {
            rc = run_sweeps(sys, chunk, 1);
            if (rc) return rc;
            done += chunk;
        }
        if (done == n_sweep && !copying) {  // spins final: copy them out while S(q) and the energy run
            if (packed) {
                pc::launch_spins_to_xyz(sys->d_stage3.p, sys->d_spins.p, n0, sys->stream);
                PC_LAUNCH_CK();
                sys->launches++;
            }
            PC_CK(cudaEventRecord(sys->ev_swept, sys->stream));
            PC_CK(cudaStreamWaitEvent(sys->copy_stream, sys->ev_swept, 0));
            PC_CK(cudaMemcpyAsync(S_out, dev_io, bytes, cudaMemcpyDeviceToHost, sys->copy_stream));
            copying = true;
        }
        if (do_ssf && chunk == ssf_every) {
            pc::SsfOut o = ssf_out_base(sys);
            o.acc_sum = sys->d_ssf_sum.p;
            o.acc_sq = sys->d_ssf_sq.p;
            o.slot_of_rep = sys->d_slot_of_rep.p;
            pc::SsfGeom geom{grp->L, grp->P, grp->Q, 1, grp->d_rep_index.p, sys->ssf_resolved ? 1 : 0};
            pc::launch_ssf_xy(geom, sys->d_spins.p, sys->d_reps.p, grp->d_G.p, sys->stream);
            PC_LAUNCH_CK();
            pc::launch_ssf_z(geom, grp->d_G.p, o, sys->stream);
            PC_LAUNCH_CK();
            sys->launches += 2;
            sys->ssf_n[size_t(ssf_slot)]++;
        }
    }
    rc = enqueue_energy(sys);
    if (rc) return rc;
    PC_CK(cudaMemcpyAsync(st_e, sys->d_e.p, sizeof(double), cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaMemcpyAsync(st_acc, sys->d_acc.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaMemcpyAsync(st_flag, sys->d_err.p, sizeof(int), cudaMemcpyDeviceToHost, sys->stream));
    PC_CK(cudaStreamSynchronize(sys->stream));
    PC_CK(cudaStreamSynchronize(sys->copy_stream));
    if (e_out) *e_out = *st_e;
    if (accepted) *accepted = *st_acc;
    return device_error_flag(sys, *st_flag);
}
}  // namespace

int pc_step_host(pc_system* sys, const float* S4_in, float* S4_out, double T, int n_sweep, int ssf_every,
                 int ssf_slot, double* e_out, uint64_t* accepted) {
    return step_host(sys, S4_in, S4_out, false, T, n_sweep, ssf_every, ssf_slot, e_out, accepted);
}

int pc_step_host3(pc_system* sys, const float* S3_in, float* S3_out, double T, int n_sweep, int ssf_every,
                  int ssf_slot, double* e_out, uint64_t* accepted) {
    return step_host(sys, S3_in, S3_out, true, T, n_sweep, ssf_every, ssf_slot, e_out, accepted);
}

int pc_set_wait_limit(pc_system* sys, int polls) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    sys->wait_polls = polls < 0 ? pc::kStagedMaxPolls : std::min(polls, pc::kStagedMaxPolls);
    sys->barrier_polls = polls < 0 ? kBarrierMaxPolls : std::min(polls, kBarrierMaxPolls);
    sys->drop_graphs();  // captured passes carry the old bound
    return PC_OK;
}

int pc_set_pt_persistent(pc_system* sys, int on) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (on) {
        rc = check_sys(sys);
        if (rc) return rc;
        if (const char* why = pt_persistent_unsupported(sys)) return fail(PC_ERR_UNSUPPORTED, why);
    }
    sys->pt_persistent = on != 0;
    return PC_OK;
}

int pc_get_pt_persistent(pc_system* sys, int* on) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    if (!on) return fail(PC_ERR_INVALID, "null output");
    *on = sys->pt_persistent ? 1 : 0;
    return PC_OK;
}

int pc_set_kernel_timing(pc_system* sys, int on) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    sys->timing = on != 0;
    sys->ev_used = 0;
    return PC_OK;
}

int pc_last_kernel_times(pc_system* sys, double* metropolis_ms, double* overrelax_ms) {
    int rc = check_sys(sys, false);
    if (rc) return rc;
    PC_CK(cudaStreamSynchronize(sys->stream));
    double tot[2] = {0, 0};
    int cnt[2] = {0, 0};
    for (size_t i = 0; i < sys->ev_used; ++i) {
        float ms = 0.f;
        PC_CK(cudaEventElapsedTime(&ms, sys->ev_pool[i].first, sys->ev_pool[i].second));
        tot[sys->ev_kind[i]] += ms;
        cnt[sys->ev_kind[i]]++;
    }
    if (metropolis_ms) *metropolis_ms = cnt[0] ? tot[0] / cnt[0] : 0.0;
    if (overrelax_ms) *overrelax_ms = cnt[1] ? tot[1] / cnt[1] : 0.0;
    sys->ev_used = 0;
    return PC_OK;
}

}  // extern "C"
