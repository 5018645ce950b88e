// fm_api.cu -- C ABI and host-side step driver of the B200 MD hot path.
//
// The driver mirrors md_advance_vv (md.f90:143-163): per iteration it queues
// move(1), the rebuild decision, the (device-gated) rebuild pipeline, forces
// and move(2), and the record reduction on tplot steps.  Move(2) of one
// iteration and move(1) of the next are fused into the force kernel, so a
// non-rebuild step is one force launch plus the small decision kernel and
// the rebuild branch.  Where CUDA graphs with conditional nodes are available
// the rebuild branch of a step is one graph launch: the decision kernel sets
// the condition of an IF node whose body holds the rebuild kernels, so a step
// without a rebuild launches the decision and the force kernel only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fm_common.cuh"
#include "fm_tile.cuh"
#include "flowmol_b200.h"

using fm::FmDev;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

#define FM_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(FM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)

#define FM_TRY(call)                 \
    do {                             \
        int r_ = (call);             \
        if (r_ != FM_OK) return r_;  \
    } while (0)

const double kPi = 3.14159265358979323846;

inline double p3(double s) { return s * s * s; }
inline double p6(double s) { double t = p3(s); return t * t; }
inline double p12(double s) { double t = p6(s); return t * t; }

}  // namespace

void fm::set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

struct fm_handle {
    fm_params p{};
    FmDev d{};
    cudaStream_t st = nullptr;
    int device = 0;
    int iter = 0;
    double simtime = 0.0;
    int stage = 0;            // 0 created, 1 state uploaded, 2 forces valid, 3 broken
    int tpm = 8;
    double half_min_delta = 0.0;
    double4 *tpos = nullptr;
    int32_t *tuidx = nullptr;
    int32_t *glob = nullptr;  // device: glob_no of upload index
    std::vector<int32_t> glob_host;
    double *stage3 = nullptr; // device staging, 3 arrays of (3, n)
    // queued fused-loop range, kept so that a list overflow can be resumed
    struct Range {
        bool active = false;
        int first_iter = 0;
        int nsteps = 0;
        std::vector<double> simtime_after;  // simtime after step k of the range
    } q;
    bool has_pe = false;
    bool cells_valid = false;  // cell_start/perm describe the current slot order
    bool list_valid = false;   // the neighbour list was built after the last re-order
    // instrumentation
    bool timing = false;
    std::vector<cudaEvent_t> ev;
    size_t ev_used = 0;
    int64_t launches = 0;
    int expected_nbr = 0;  // (4/3) pi r_n^3 rho, rounded: the autotuner's key
    int cap = 0;           // molecules the arrays hold: np, or a subdomain's capacity
    // subdomain of a spatial decomposition (d.dd = 1)
    fm::DdDev x{};
    int nranks = 0;
    bool planned = false;
    int n_own = 0, n_halo = 0;  // after the last sort: owned molecules and halo copies (d.n = both)
    int n_kept = 0;             // owned molecules kept by the last classification
    int n_pending = 0;          // array entries before the sort (old entries + arrivals)
    int dd_phase = 0;           // rebuild: 0 idle, 1 classified, 2 immigrated, 3 halo counted
    int32_t *dd_dev = nullptr;  // device block behind x (plan and counters)
    double *dd_sums = nullptr;  // device [RS_N]
    std::vector<int32_t> dd_counts;
    // rebuild branch as a CUDA graph, per `flip` (whether the previous force
    // kernel already did this step's move(1)); rebuilt when the device state
    // it was captured with (FmDev) changes
    // [flip] rebuild branch, [2 + flip] STEP_GRAPH_K whole iterations
    cudaGraphExec_t rbx[4] = {nullptr, nullptr, nullptr, nullptr};
    FmDev rbd[4]{};
    int rbt[4] = {0, 0, 0, 0};    // lanes per molecule the force kernels were captured with
    bool rb_off = false;          // graphs unavailable here: per-kernel launches
    cudaStream_t cap_st = nullptr, cap_st2 = nullptr, cap_st3 = nullptr;
    // sort_mols (fm_sort.cu): sort_flag 0 leaves the numbering alone
    int sort_flag = 0;
    fm::FmSortDev sdev{};
    bool glob_moved = false;      // a sort was configured: global numbers live on the device
};

// ---------------------------------------------------------------------------
// geometry (setup_set_parameters.f90)
// ---------------------------------------------------------------------------

// rcutoff after set_parameters_cells: with the Soddemann solvent a rneighbr
// below sod_cut raises it to sod_cut (:1871-1876), which the cells, potshift
// (:1222) and the long-range corrections (:1226-1238) then use.
static double effective_rcutoff(const fm_params *p)
{
    const double rneighbr = p->rcutoff + (p->delta_rneighbr[0] + p->delta_rneighbr[1] + p->delta_rneighbr[2]) / 3.0;
    return p->potential_flag == 1 && p->solvent_flag == 1 && rneighbr < fm::SOD_CUT ? fm::SOD_CUT : p->rcutoff;
}

static int derive(const fm_params *p, int32_t nc[3], double cs[3], double *rn2, double *rc2, double *ps)
{
    if (!p) return fail(FM_ERR_ARG, "null params");
    if (!(p->rcutoff > 0.0)) return fail(FM_ERR_ARG, "rcutoff must be > 0");
    for (int k = 0; k < 3; k++)
        if (!(p->domain[k] > 0.0)) return fail(FM_ERR_ARG, "domain must be > 0");
    // rneighbr = rcutoff + mean(delta) (set_parameters_cells :1858-1859)
    double rneighbr = p->rcutoff + (p->delta_rneighbr[0] + p->delta_rneighbr[1] + p->delta_rneighbr[2]) / 3.0;
    double rneighbr2 = rneighbr * rneighbr;
    if (p->potential_flag == 1 && p->solvent_flag == 0 && rneighbr < p->R_0)
        rneighbr2 = p->R_0 * p->R_0;  // :1865-1869
    const double rcutoff = effective_rcutoff(p);  // rneighbr2 stays with the Soddemann raise
    for (int k = 0; k < 3; k++) nc[k] = (int32_t)std::floor(p->domain[k] / (rcutoff + p->delta_rneighbr[k]));
    *rn2 = rneighbr2;
    *rc2 = rcutoff * rcutoff;
    *ps = 4.0 * (1.0 / p12(rcutoff) - 1.0 / p6(rcutoff));  // :1222
    bool few = nc[0] < 3 || nc[1] < 3 || nc[2] < 3;
    for (int k = 0; k < 3; k++) cs[k] = nc[k] > 0 ? p->domain[k] / (double)nc[k] : p->domain[k];
    if (few) return fail(FM_ERR_FEWCELLS, "domain should have at least 3 cells in x, y and z");
    return FM_OK;
}

extern "C" int fm_derive_geometry(const fm_params *p, int32_t ncells[3], double cellsidelength[3],
                                  double *rneighbr2, double *rcutoff2, double *potshift)
{
    if (!ncells || !cellsidelength || !rneighbr2 || !rcutoff2 || !potshift) return fail(FM_ERR_ARG, "null output");
    return derive(p, ncells, cellsidelength, rneighbr2, rcutoff2, potshift);
}

extern "C" int fm_global_domain(const int32_t nunits[3], double density, double domain[3])
{
    if (!nunits || !domain || !(density > 0.0)) return fail(FM_ERR_ARG, "bad arguments");
    for (int k = 0; k < 3; k++) domain[k] = (double)nunits[k] / std::pow(density / 4.0, 1.0 / 3.0);
    return FM_OK;
}

extern "C" int fm_last_error(char *buf, int32_t len)
{
    if (!buf || len <= 0) return FM_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", g_last_error.c_str());
    return FM_OK;
}

// ---------------------------------------------------------------------------
// allocation
// ---------------------------------------------------------------------------

template <typename T>
static int dalloc(T **ptr, size_t count)
{
    *ptr = nullptr;
    if (count == 0) count = 1;
    FM_CUDA(cudaMalloc((void **)ptr, count * sizeof(T)));
    return FM_OK;
}

static void release_graphs(fm_handle *h)
{
    for (int f = 0; f < 4; f++) {
        if (h->rbx[f]) cudaGraphExecDestroy(h->rbx[f]);
        h->rbx[f] = nullptr;
    }
}

// Kernels of one launch_sort (the radix sort's own are the library's).
constexpr int SORT_KERNELS = 5;

static void free_sort(fm_handle *h)
{
    fm::FmSortDev &s = h->sdev;
    void *ptrs[] = {(void *)s.hc, s.key, s.key_out, s.val, s.val_out, s.cnt, s.newv, s.gtmp, s.tmp, s.ss};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    s = fm::FmSortDev{};
    h->sort_flag = 0;
}

static void release(fm_handle *h)
{
    release_graphs(h);
    free_sort(h);
    if (h->cap_st) cudaStreamDestroy(h->cap_st);
    if (h->cap_st2) cudaStreamDestroy(h->cap_st2);
    if (h->cap_st3) cudaStreamDestroy(h->cap_st3);
    h->cap_st = h->cap_st2 = h->cap_st3 = nullptr;
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    h->ev.clear();
    FmDev &d = h->d;
    void *ptrs[] = {d.pos0, d.pos1, d.vx, d.vy, d.vz, d.ax, d.ay, d.az, d.slot_of, d.tvx, d.tvy, d.tvz,
                    d.tax, d.tay, d.taz, d.cell_of, d.cell_count, d.cell_start, d.perm, d.tile_sum, d.nbr, d.nnbr,
                    d.pe, d.vir, d.partial, d.rec, d.sc, h->tpos, h->tuidx, h->glob, h->stage3, d.chain,
                    d.subchain, d.bflag, d.tchain, d.tsubchain, d.tbflag, d.bnd, d.nbond,
                    (void *)d.mie_pair, (void *)d.mie_mass, (void *)d.mie_type_up, d.rdx, d.rdy, d.rdz, d.rf6,
                    d.blk_off, d.nbr16, (void *)d.ang_k, (void *)d.ang_t0, d.funcy, d.tfuncy, h->dd_dev,
                    h->dd_sums};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    d = FmDev{};
    h->tpos = nullptr; h->tuidx = nullptr; h->glob = nullptr; h->stage3 = nullptr;
    h->dd_dev = nullptr; h->dd_sums = nullptr;
}

static int pick_tpm(const fm_params &p, double expected_full)
{
    if (p.threads_per_molecule > 0) {
        int t = p.threads_per_molecule;
        if (t != 1 && t != 2 && t != 4 && t != 8 && t != 16) return -1;
        return t;
    }
    // about 8-12 candidates per lane keeps the lanes of a group busy while the
    // shuffle reduction stays short
    if (expected_full > 96) return 8;
    if (expected_full > 40) return 4;
    if (expected_full > 16) return 2;
    return 1;
}

static int round_up(int x, int m) { return ((x + m - 1) / m) * m; }

static int alloc_nlist(fm_handle *h, int maxn)
{
    FmDev &d = h->d;
    maxn = round_up(std::max(maxn, 8), 8);  // 16-byte aligned rows for the vector reads
    if (d.nbr) cudaFree(d.nbr);
    d.nbr = nullptr;
    d.maxn = maxn;
    FM_TRY(dalloc(&d.nbr, fm::nb_rows(h->cap) * (size_t)maxn));
    return FM_OK;
}

// Rows of the tiled path: a multiple of 8 T entries (one 16-byte load per
// lane per chunk).
static int alloc_nlist16(fm_handle *h, int maxn)
{
    FmDev &d = h->d;
    maxn = round_up(std::max(maxn, 8 * d.tile_T), 8 * d.tile_T);
    if (d.nbr16) cudaFree(d.nbr16);
    d.nbr16 = nullptr;
    d.maxn16 = maxn;
    FM_TRY(dalloc(&d.nbr16, (size_t)h->cap * (size_t)maxn));
    return FM_OK;
}

// Leaves the tiled path for the per-entry gather path (a block's staged
// neighbourhood would no longer fit in shared memory): generic rows of the
// same capacity; the caller builds them.
static int leave_tiles(fm_handle *h)
{
    FmDev &d = h->d;
    const int maxn = d.maxn16;
    if (d.nbr16) cudaFree(d.nbr16);
    d.nbr16 = nullptr;
    d.tile = 0;
    FM_TRY(alloc_nlist(h, maxn));
    return FM_OK;
}

// Record partial rows the force kernel writes: one per CTA, or one per block
// on the tiled path.
static int force_rows(const fm_handle *h)
{
    return h->d.tile ? h->d.tile_nblk : fm::force_blocks(h->d.n, h->tpm);
}

// The list build of a rebuild: on the tiled path the blocks' staging table
// first, then the rows.
static void queue_build(fm_handle *h, int gated, int iter)
{
    if (h->d.tile) { fm::launch_blk_seg(h->d, gated, iter, h->st); h->launches += 1; }
    fm::launch_build_nlist(h->d, gated, iter, h->st);
    if (h->d.angular) { fm::launch_angular_order(h->d, gated, iter, h->st); h->launches += 1; }
}

// A subdomain's block of the undivided system's cells (fm_dd_create).
struct DdGeom {
    int32_t nglob[3], org[3], nloc[3];
    int32_t capacity;
};

static int create_impl(const fm_params *p, const DdGeom *g, fm_handle **out)
{
    if (!p || !out) return fail(FM_ERR_ARG, "null argument");
    *out = nullptr;
    if (p->np <= 0 || p->np > fm::MAX_MOLECULES) return fail(FM_ERR_ARG, "np out of range (1 .. 2^26-1)");
    if (p->tplot <= 0) return fail(FM_ERR_ARG, "tplot must be > 0");
    if (!(p->delta_t > 0.0)) return fail(FM_ERR_ARG, "delta_t must be > 0");
    if (p->force_list != 0 && p->force_list != 2 && p->force_list != 3)
        return fail(FM_ERR_ARG, "force_list must be 0, 2 or 3");
    if (p->list_build != FM_LIST_BUILD_AUTO && p->list_build != FM_LIST_BUILD_CELLS &&
        p->list_build != FM_LIST_BUILD_BLOCKS)
        return fail(FM_ERR_ARG, "list_build must be FM_LIST_BUILD_AUTO, _CELLS or _BLOCKS");
    if (p->precision != FM_PRECISION_FP64 && p->precision != FM_PRECISION_FP32)
        return fail(FM_ERR_ARG, "precision must be FM_PRECISION_FP64 or FM_PRECISION_FP32");
    if (p->potential_flag != 0 && p->potential_flag != 1) return fail(FM_ERR_ARG, "potential_flag must be 0 or 1");
    if (p->potential_flag == 1 && p->force_list == 0)
        return fail(FM_ERR_ARG, "potential flag/force_list incompatible - only LJ available with all pairs");
    if (p->potential_flag == 1 && p->force_list == 2)  // simulation_compute_forces.f90:242-246
        return fail(FM_ERR_ARG,
                    "potential flag/force_list incompatible - only LJ available with full interaction neighbour lists");
    if (p->potential_flag == 1 && !(p->R_0 > 0.0 && p->k_c >= 0.0)) return fail(FM_ERR_ARG, "FENE needs R_0 > 0");
    if (p->solvent_flag != 0 && p->solvent_flag != 1) return fail(FM_ERR_ARG, "solvent_flag must be 0 or 1");
    if (p->solvent_flag == 1 && (p->potential_flag != 1 || p->force_list != 3))
        return fail(FM_ERR_ARG, "the Soddemann solvent (solvent_flag 1) needs potential_flag 1 and force_list 3");
    if (p->rebuild_criteria < 0 || p->rebuild_criteria > 2)
        return fail(FM_ERR_ARG, "rebuild_criteria must be 0 (vmax), 1 (fixed) or 2 (displacement)");
    if (p->integration_algorithm != 0 && p->integration_algorithm != 1)
        return fail(FM_ERR_ARG, "integration_algorithm must be 0 (leap-frog) or 1 (velocity Verlet)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FM_ERR_NODEVICE, "no CUDA device");

    int32_t nc[3];
    double cs[3], rn2, rc2, ps;
    int grc = derive(p, nc, cs, &rn2, &rc2, &ps);
    if (grc != FM_OK && !(grc == FM_ERR_FEWCELLS && p->force_list == 0)) return grc;
    if (g) {
        // subdomain: the LJ neighbour-list path with velocity Verlet and rebuild
        // criteria 0/1, per-entry gather kernel
        if (p->force_list == 0) return fail(FM_ERR_ARG, "a subdomain needs a neighbour list (force_list 2 or 3)");
        if (p->potential_flag != 0 || p->solvent_flag != 0)
            return fail(FM_ERR_ARG, "a subdomain runs the LJ/WCA pair potential (potential_flag 0)");
        if (p->integration_algorithm != 1) return fail(FM_ERR_ARG, "a subdomain integrates with velocity Verlet");
        if (p->rebuild_criteria != 0 && p->rebuild_criteria != 1)
            return fail(FM_ERR_ARG, "a subdomain takes rebuild_criteria 0 (vmax) or 1 (fixed)");
        if (p->force_path == FM_FORCE_PATH_TILES) return fail(FM_ERR_ARG, "a subdomain uses the gather force path");
        for (int k = 0; k < 3; k++) {
            if (g->nglob[k] != nc[k])
                return fail(FM_ERR_ARG, "ncells_global differs from the cells fm_derive_geometry gives");
            if (g->nloc[k] < 1 || g->org[k] < 0 || g->org[k] + g->nloc[k] > g->nglob[k])
                return fail(FM_ERR_ARG, "subdomain cells outside the global grid");
        }
        if (g->capacity < 1 || g->capacity > fm::MAX_MOLECULES) return fail(FM_ERR_ARG, "capacity out of range");
    }

    fm_handle *h = new fm_handle();
    h->p = *p;
    FM_CUDA(cudaGetDevice(&h->device));
    FmDev &d = h->d;
    d.n = g ? 0 : p->np;
    h->cap = g ? g->capacity : p->np;
    for (int k = 0; k < 3; k++) {
        d.L[k] = p->domain[k];
        d.hd[k] = 0.5 * p->domain[k];
        d.cs[k] = cs[k];
        d.nc[k] = p->force_list == 0 ? 1 : (g ? g->nloc[k] : nc[k]);
        d.ne[k] = d.nc[k] + 2;
        if (g) { d.org[k] = g->org[k]; d.gne[k] = g->nglob[k] + 2; }
    }
    d.dd = g ? 1 : 0;
    d.ncell = d.ne[0] * d.ne[1] * d.ne[2];
    d.rc2 = rc2;
    d.rn2 = rn2;
    d.dt = p->delta_t;
    d.half_dt = 0.5 * p->delta_t;
    d.half_dt2 = 0.5 * (p->delta_t * p->delta_t);
    d.potshift = ps;
    d.density = p->density > 0.0 ? p->density : (double)p->np / (p->domain[0] * p->domain[1] * p->domain[2]);
    if (p->sLRC_flag) {  // setup_set_parameters.f90:1226-1238
        const double rc = effective_rcutoff(p);
        d.pot_slrc = 8.0 * kPi * d.density * (1.0 / (9.0 * std::pow(rc, 9)) - 1.0 / (3.0 * p3(rc)));
        d.p_slrc = 8.0 * kPi * std::pow(d.density, 2.0) * (4.0 / (9.0 * std::pow(rc, 9)) - 2.0 / (3.0 * p3(rc)));
    }
    d.tplot = p->tplot;
    d.integrator = p->integration_algorithm;
    d.potential_flag = p->potential_flag;
    d.solvent = p->potential_flag == 1 && p->solvent_flag == 1 ? 1 : 0;
    d.sod_eps[0] = p->eps_ss; d.sod_eps[1] = p->eps_ps; d.sod_eps[2] = p->eps_pp;
    d.k_c = p->k_c;
    d.R0 = p->R_0;
    d.R0_2 = p->R_0 * p->R_0;
    d.precision = p->precision;
    double dmin = std::min(p->delta_rneighbr[0], std::min(p->delta_rneighbr[1], p->delta_rneighbr[2]));
    h->half_min_delta = 0.5 * dmin;

    double rho = (double)p->np / (p->domain[0] * p->domain[1] * p->domain[2]);
    double expected = 4.0 / 3.0 * kPi * std::pow(std::sqrt(rn2), 3) * std::max(rho, 0.25);
    // sparse cells (a few molecules each) are built 2x2x2 at a time: same rows,
    // the per-cell latency shared by eight cells
    const double per_cell = rho * d.cs[0] * d.cs[1] * d.cs[2];
    d.build_blocks = p->list_build == FM_LIST_BUILD_BLOCKS ? 1
                     : p->list_build == FM_LIST_BUILD_CELLS ? 0 : (per_cell < 8.0 ? 1 : 0);
    int tpm = pick_tpm(*p, expected);
    if (g && p->threads_per_molecule == 0) h->p.threads_per_molecule = tpm;  // every rank the same kernel
    if (tpm < 0) { delete h; return fail(FM_ERR_ARG, "threads_per_molecule must be 0, 1, 2, 4, 8 or 16"); }
    if (p->force_path != FM_FORCE_PATH_AUTO && p->force_path != FM_FORCE_PATH_GATHER &&
        p->force_path != FM_FORCE_PATH_TILES) {
        delete h;
        return fail(FM_ERR_ARG, "force_path must be FM_FORCE_PATH_AUTO, _GATHER or _TILES");
    }
    // tiled force path: dense systems (the list build's own choice of one warp
    // per cell), lanes per molecule 4 or 8; a staged neighbourhood of 64 cells
    // must fit in shared memory
    {
        const bool tpm_ok = p->threads_per_molecule == 0 || p->threads_per_molecule == 4 ||
                            p->threads_per_molecule == 8;
        const double est_union = 64.0 * std::max(per_cell, 0.25);
        const bool fits = 1.25 * est_union + 64.0 < (double)fm::tile_ucap_limit(3);
        // automatic keeps the gather kernel: on the 1M LJ liquid the tiled kernel
        // measured 0.29-0.30 ms against 0.28 ms (its shared-memory reads are
        // bank-conflicted and the neighbourhood is staged eight times); the
        // tiled rows take half the list memory
        const bool want = p->force_list != 0 && tpm_ok && fits && p->force_path == FM_FORCE_PATH_TILES;
        if (p->force_path == FM_FORCE_PATH_TILES && !want) {
            delete h;
            return fail(FM_ERR_ARG, "force_path TILES needs a neighbour list, threads_per_molecule 0, 4 or 8, "
                                    "and a 4x4x4-cell neighbourhood that fits in shared memory");
        }
        if (want) {
            d.tile = 1;
            d.tile_T = p->threads_per_molecule == 4 ? 4 : p->threads_per_molecule == 8 ? 8 : (expected > 24 ? 8 : 4);
            d.tile_R = 3;  // (4 once Mie types or Soddemann bead flags are set; fixed at fm_setup)
            for (int k = 0; k < 3; k++) d.tile_nb[k] = (d.ne[k] + 1) / 2;
            d.tile_nblk = d.tile_nb[0] * d.tile_nb[1] * d.tile_nb[2];
            d.tile_ucap = std::min(round_up((int)std::ceil(1.25 * est_union) + 64, 32), fm::tile_ucap_limit(3));
            tpm = d.tile_T;
        }
    }
    h->tpm = tpm;
    // FM_STEP_GRAPHS=0: every kernel of a step is launched on its own (the
    // same kernels and results); Nsight Compute does not profile kernel nodes
    // of graphs that hold conditional nodes
    if (const char *e = std::getenv("FM_STEP_GRAPHS")) h->rb_off = std::strcmp(e, "0") == 0;
    h->expected_nbr = (int)std::lround(expected);
    int maxn = p->nlist_capacity > 0 ? p->nlist_capacity : round_up((int)std::ceil(1.3 * expected) + 16, 8);

    const size_t n = (size_t)h->cap;
    int rc = FM_OK;
#define FM_ALLOC(ptr, cnt)                                   \
    if (rc == FM_OK) rc = dalloc(&(ptr), (size_t)(cnt));
    FM_ALLOC(d.pos0, n) FM_ALLOC(d.pos1, n)
    FM_ALLOC(d.vx, n) FM_ALLOC(d.vy, n) FM_ALLOC(d.vz, n)
    FM_ALLOC(d.ax, n) FM_ALLOC(d.ay, n) FM_ALLOC(d.az, n)
    FM_ALLOC(d.tvx, n) FM_ALLOC(d.tvy, n) FM_ALLOC(d.tvz, n)
    FM_ALLOC(d.tax, n) FM_ALLOC(d.tay, n) FM_ALLOC(d.taz, n)
    FM_ALLOC(d.slot_of, n) FM_ALLOC(h->tuidx, n) FM_ALLOC(h->tpos, n) FM_ALLOC(h->glob, n)
    FM_ALLOC(d.cell_of, n) FM_ALLOC(d.perm, n) FM_ALLOC(d.nnbr, n)
    FM_ALLOC(d.cell_count, d.ncell) FM_ALLOC(d.cell_start, d.ncell + 1)
    FM_ALLOC(d.tile_sum, fm::scan_tiles(d.ncell))
    FM_ALLOC(d.pe, n) FM_ALLOC(d.vir, n)
    FM_ALLOC(h->stage3, 9 * n)
    if (p->rebuild_criteria == 2) { FM_ALLOC(d.rdx, n) FM_ALLOC(d.rdy, n) FM_ALLOC(d.rdz, n) }
    if (p->potential_flag == 1) {
        FM_ALLOC(d.chain, n) FM_ALLOC(d.subchain, n) FM_ALLOC(d.bflag, n)
        FM_ALLOC(d.tchain, n) FM_ALLOC(d.tsubchain, n) FM_ALLOC(d.tbflag, n)
        FM_ALLOC(d.bnd, 4 * n) FM_ALLOC(d.nbond, n)
    }
    int nb = std::max(std::max(fm::force_blocks(h->cap, 16), fm::all_pairs_blocks(h->cap)), fm::macro_blocks(h->cap));
    nb = std::max(nb, d.tile_nblk);
    if (d.tile) { FM_ALLOC(d.blk_off, (size_t)d.tile_nblk * fm::TILE_NSEGP) }
    FM_ALLOC(d.partial, (size_t)nb * fm::RS_N)
    d.rec_cap = 4096;
    FM_ALLOC(d.rec, d.rec_cap)
    FM_ALLOC(d.sc, 1)
#undef FM_ALLOC
    if (rc == FM_OK && p->force_list != 0) rc = d.tile ? alloc_nlist16(h, maxn) : alloc_nlist(h, maxn);
    if (rc != FM_OK) {
        std::string msg = g_last_error;
        release(h);
        delete h;
        return fail(rc, msg);
    }
    d.nblocks_force = force_rows(h);
    cudaMemset(d.cell_count, 0, sizeof(int32_t) * (size_t)d.ncell);
    cudaMemset(d.cell_start, 0, sizeof(int32_t) * (size_t)(d.ncell + 1));
    cudaMemset(d.nnbr, 0, sizeof(int32_t) * n);
    cudaMemset(d.pe, 0, sizeof(double) * n);
    if (d.nbond) cudaMemset(d.nbond, 0, sizeof(int32_t) * n);
    if (d.chain) cudaMemset(d.chain, 0, sizeof(int32_t) * n);
    if (d.subchain) cudaMemset(d.subchain, 0, sizeof(int32_t) * n);
    if (d.bflag) cudaMemset(d.bflag, 0, sizeof(int4) * n);
    cudaMemset(d.vir, 0, sizeof(double) * n);
    cudaMemset(d.sc, 0, sizeof(fm::FmScalars));
    fm::launch_reset_scalars(d, nullptr);
    FM_CUDA(cudaGetLastError());
    FM_CUDA(cudaDeviceSynchronize());
    h->iter = p->initialstep;
    h->simtime = p->simtime;
    *out = h;
    return FM_OK;
}

extern "C" int fm_create(const fm_params *p, fm_handle **out) { return create_impl(p, nullptr, out); }

extern "C" int fm_destroy(fm_handle *h)
{
    if (!h) return FM_OK;
    cudaStreamSynchronize(h->st);
    release(h);
    delete h;
    return FM_OK;
}

extern "C" int fm_set_stream(fm_handle *h, void *stream)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    h->st = (cudaStream_t)stream;
    return FM_OK;
}

// ---------------------------------------------------------------------------
// state transfer
// ---------------------------------------------------------------------------

static int begin_state(fm_handle *h, int32_t n)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (h->d.dd) return fail(FM_ERR_STATE, "a subdomain handle takes its molecules through fm_dd_upload");
    if (n != h->d.n) return fail(FM_ERR_ARG, "n differs from the np the handle was created with");
    h->q.active = false;
    h->cells_valid = false;
    h->list_valid = false;
    h->iter = h->p.initialstep;
    h->simtime = h->p.simtime;
    h->d.nblocks_force = force_rows(h);
    fm::launch_reset_scalars(h->d, h->st);
    FM_CUDA(cudaMemsetAsync(h->d.cell_count, 0, sizeof(int32_t) * (size_t)h->d.ncell, h->st));
    return FM_OK;
}

static int set_glob(fm_handle *h, const int32_t *glob_no)
{
    const int n = h->d.n;
    h->glob_host.resize((size_t)n);
    for (int i = 0; i < n; i++) h->glob_host[(size_t)i] = glob_no ? glob_no[i] : i + 1;
    FM_CUDA(cudaMemcpyAsync(h->glob, h->glob_host.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, h->st));
    return FM_OK;
}

extern "C" int fm_upload_state(fm_handle *h, int32_t n, const double *r, const double *v, const double *a,
                               const int32_t *glob_no)
{
    FM_TRY(begin_state(h, n));
    if (!r || !v) return fail(FM_ERR_ARG, "r and v are required");
    const size_t bytes = sizeof(double) * 3 * (size_t)n;
    double *dr = h->stage3, *dv = h->stage3 + 3 * (size_t)n, *da = h->stage3 + 6 * (size_t)n;
    FM_CUDA(cudaMemcpyAsync(dr, r, bytes, cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaMemcpyAsync(dv, v, bytes, cudaMemcpyHostToDevice, h->st));
    if (a) FM_CUDA(cudaMemcpyAsync(da, a, bytes, cudaMemcpyHostToDevice, h->st));
    fm::launch_scatter_state(h->d, dr, dv, a ? da : nullptr, h->st);
    FM_TRY(set_glob(h, glob_no));
    FM_CUDA(cudaGetLastError());
    FM_CUDA(cudaStreamSynchronize(h->st));
    h->stage = 1;
    return FM_OK;
}

extern "C" int fm_upload_state_device(fm_handle *h, int32_t n, const double *d_r, const double *d_v)
{
    FM_TRY(begin_state(h, n));
    if (!d_r || !d_v) return fail(FM_ERR_ARG, "r and v are required");
    fm::launch_scatter_state(h->d, d_r, d_v, nullptr, h->st);
    FM_TRY(set_glob(h, nullptr));
    FM_CUDA(cudaGetLastError());
    h->stage = 1;
    return FM_OK;
}

extern "C" int fm_upload_monomers(fm_handle *h, const int32_t *chainID, const int32_t *subchainID,
                                  const int32_t *bin_bflag)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (h->p.potential_flag != 1) return fail(FM_ERR_STATE, "monomer data needs potential_flag 1");
    if (h->stage != 1) return fail(FM_ERR_STATE, "upload monomers after fm_upload_state and before fm_setup");
    if (!chainID || !subchainID || !bin_bflag) return fail(FM_ERR_ARG, "null array");
    const size_t n = (size_t)h->d.n;
    // slots still equal upload indices before the first binning
    FM_CUDA(cudaMemcpyAsync(h->d.chain, chainID, 4 * n, cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaMemcpyAsync(h->d.subchain, subchainID, 4 * n, cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaMemcpyAsync(h->d.bflag, bin_bflag, 16 * n, cudaMemcpyHostToDevice, h->st));
    if (h->d.solvent) fm::launch_set_bead_flags(h->d, h->st);
    FM_CUDA(cudaGetLastError());
    FM_CUDA(cudaStreamSynchronize(h->st));
    return FM_OK;
}

static int ready(fm_handle *h, int min_stage);

extern "C" int fm_set_angular(fm_handle *h, int32_t ntypes, const double *k_lookup, const double *theta0_lookup,
                              const int32_t *funcy)
{
    if (!h || !k_lookup || !theta0_lookup || !funcy) return fail(FM_ERR_ARG, "null argument");
    if (h->stage != 1) return fail(FM_ERR_STATE, "set the angular tables after fm_set_mie and before fm_setup");
    const fm_params &p = h->p;
    if (p.force_list != 3 || p.potential_flag != 1 || p.solvent_flag != 0)
        return fail(FM_ERR_ARG, "angular_potential needs force_list 3, potential_flag 1 and solvent_flag 0 "
                                "(simulation_compute_forces.f90:257-259)");
    FmDev &d = h->d;
    if (!d.mie) return fail(FM_ERR_STATE, "angular_potential looks up the Mie types: call fm_set_mie first");
    if (ntypes < 1 || ntypes > FM_MIE_MAXTYPES) return fail(FM_ERR_ARG, "ntypes out of range (1 .. FM_MIE_MAXTYPES)");
    const size_t n3 = (size_t)ntypes * ntypes * ntypes, n = (size_t)d.n;
    for (size_t u = 0; u < n; u++)
        if (funcy[u] < 0 || funcy[u] > 4) return fail(FM_ERR_ARG, "funcy out of range (0 .. 4)");
    if (!d.funcy) {
        FM_TRY(dalloc(&d.funcy, n));
        FM_TRY(dalloc(&d.tfuncy, n));
        double *k = nullptr, *t = nullptr;
        FM_TRY(dalloc(&k, (size_t)FM_MIE_MAXTYPES * FM_MIE_MAXTYPES * FM_MIE_MAXTYPES));
        d.ang_k = k;
        FM_TRY(dalloc(&t, (size_t)FM_MIE_MAXTYPES * FM_MIE_MAXTYPES * FM_MIE_MAXTYPES));
        d.ang_t0 = t;
    }
    int32_t *fu = nullptr;
    FM_TRY(dalloc(&fu, n));
    cudaError_t ce = cudaMemcpyAsync(fu, funcy, sizeof(int32_t) * n, cudaMemcpyHostToDevice, h->st);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync((void *)d.ang_k, k_lookup, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync((void *)d.ang_t0, theta0_lookup, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st);
    if (ce == cudaSuccess) {
        fm::launch_set_funcy(d, fu, h->st);  // slots still equal upload indices before the first binning
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->st);
    cudaFree(fu);
    FM_CUDA(ce);
    d.ang_nt = ntypes;
    d.angular = 1;
    return FM_OK;
}

extern "C" int fm_set_mie(fm_handle *h, const fm_mie_tables *t, const int32_t *moltype)
{
    if (!h || !t || !moltype) return fail(FM_ERR_ARG, "null argument");
    if (h->stage != 1) return fail(FM_ERR_STATE, "set the Mie tables after fm_upload_state and before fm_setup");
    if (h->sort_flag) return fail(FM_ERR_ARG, "Sort should be turned off - Not developed for Mie potential");
    const int nt = t->ntypes;
    if (nt < 1 || nt > FM_MIE_MAXTYPES) return fail(FM_ERR_ARG, "ntypes out of range (1 .. FM_MIE_MAXTYPES)");
    if (!t->mass || !t->epsilon || !t->lambdar || !t->lambdaa || !t->C || !t->alpha || !t->potshift ||
        !t->k_harmonic || !t->r0)
        return fail(FM_ERR_ARG, "null table");
    for (int a = 0; a < nt; a++)
        if (!(t->mass[a] > 0.0)) return fail(FM_ERR_ARG, "mass_lookup must be > 0");
    const size_t n = (size_t)h->d.n;
    for (size_t u = 0; u < n; u++)
        if (moltype[u] < 1 || moltype[u] > nt) return fail(FM_ERR_ARG, "moltype out of range (1 .. ntypes)");
    // the reference's evaluation order, precombined per type pair (Mie_accijmag,
    // Mie_energy, harmonic_*: setup_set_parameters.f90:149-204, 384-437)
    std::vector<fm::FmMiePair> pairs((size_t)fm::MIE_MAXT * fm::MIE_MAXT);
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) {
            const size_t q = (size_t)a + (size_t)nt * (size_t)b;
            fm::FmMiePair &m = pairs[(size_t)a + (size_t)fm::MIE_MAXT * (size_t)b];
            m.ceps = t->C[q] * t->epsilon[q];
            m.lr = t->lambdar[q];
            m.ala = t->alpha[q] * t->lambdaa[q];
            m.er1 = 0.5 * t->lambdar[q] + 1.0;
            m.ea1 = 0.5 * t->lambdaa[q] + 1.0;
            m.er = 0.5 * t->lambdar[q];
            m.ea = 0.5 * t->lambdaa[q];
            m.alpha = t->alpha[q];
            m.shift = t->potshift[q];
            m.k = t->k_harmonic[q];
            m.r0 = t->r0[q];
        }
    std::vector<double> mass(fm::MIE_MAXT, 1.0);
    for (int a = 0; a < nt; a++) mass[(size_t)a] = t->mass[a];
    FmDev &d = h->d;
    if (!d.mie_pair) {
        fm::FmMiePair *dp = nullptr;
        double *dm = nullptr;
        int32_t *dt = nullptr;
        FM_CUDA(cudaMalloc(&dp, sizeof(fm::FmMiePair) * pairs.size()));
        d.mie_pair = dp;
        FM_CUDA(cudaMalloc(&dm, sizeof(double) * mass.size()));
        d.mie_mass = dm;
        FM_CUDA(cudaMalloc(&dt, sizeof(int32_t) * n));
        d.mie_type_up = dt;
    }
    FM_CUDA(cudaMemcpyAsync((void *)d.mie_pair, pairs.data(), sizeof(fm::FmMiePair) * pairs.size(),
                            cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaMemcpyAsync((void *)d.mie_mass, mass.data(), sizeof(double) * mass.size(), cudaMemcpyHostToDevice,
                            h->st));
    FM_CUDA(cudaMemcpyAsync((void *)d.mie_type_up, moltype, sizeof(int32_t) * n, cudaMemcpyHostToDevice, h->st));
    d.mie = 1;
    fm::launch_set_types(d, h->st);  // slots still equal upload indices before the first binning
    FM_CUDA(cudaGetLastError());
    FM_CUDA(cudaStreamSynchronize(h->st));
    return FM_OK;
}


extern "C" int fm_get_bonds(fm_handle *h, int32_t *owner, int32_t *partner, int8_t *code, int64_t cap, int64_t *n_out)
{
    FM_TRY(ready(h, 2));
    if (!n_out) return fail(FM_ERR_ARG, "null output");
    if (h->p.potential_flag != 1) { *n_out = 0; return FM_OK; }
    const size_t n = (size_t)h->d.n;
    std::vector<int32_t> nb(n), slot(n), bnd(4 * n);
    FM_CUDA(cudaMemcpyAsync(nb.data(), h->d.nbond, 4 * n, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaMemcpyAsync(slot.data(), h->d.slot_of, 4 * n, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaMemcpyAsync(bnd.data(), h->d.bnd, 16 * n, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    int64_t k = 0;
    for (size_t i = 0; i < n; i++)
        for (int b = 0; b < nb[i]; b++) {
            int32_t e = bnd[4 * i + (size_t)b];
            int32_t j = e & fm::NB_INDEX_MASK;
            int c6 = (int)((uint32_t)e >> fm::NB_SHIFT_BITS);
            if (k < cap) {
                if (owner) owner[k] = h->glob_host[(size_t)slot[i]];
                if (partner) partner[k] = h->glob_host[(size_t)slot[(size_t)j]];
                if (code) code[k] = (int8_t)((c6 & 3) + 3 * ((c6 >> 2) & 3) + 9 * ((c6 >> 4) & 3));
            }
            k++;
        }
    *n_out = k;
    return FM_OK;
}

// Global numbers by upload index: once a sort was configured they are
// renumbered on the device, and the host copy is refreshed before each use.
static int pull_glob(fm_handle *h)
{
    if (!h->glob_moved || h->glob_host.empty()) return FM_OK;
    FM_CUDA(cudaMemcpyAsync(h->glob_host.data(), h->glob, sizeof(int32_t) * h->glob_host.size(),
                            cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    return FM_OK;
}

extern "C" int fm_download_state(fm_handle *h, double *r, double *v, double *a, int32_t *glob_no)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (h->stage < 1) return fail(FM_ERR_STATE, "no state uploaded");
    const size_t n = (size_t)h->d.n;
    const size_t bytes = sizeof(double) * 3 * n;
    double *dr = h->stage3, *dv = h->stage3 + 3 * n, *da = h->stage3 + 6 * n;
    fm::launch_gather_state(h->d, r ? dr : nullptr, v ? dv : nullptr, a ? da : nullptr, nullptr, nullptr, nullptr,
                            h->st);
    if (r) FM_CUDA(cudaMemcpyAsync(r, dr, bytes, cudaMemcpyDeviceToHost, h->st));
    if (v) FM_CUDA(cudaMemcpyAsync(v, dv, bytes, cudaMemcpyDeviceToHost, h->st));
    if (a) FM_CUDA(cudaMemcpyAsync(a, da, bytes, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaGetLastError());
    FM_CUDA(cudaStreamSynchronize(h->st));
    if (glob_no) {
        FM_TRY(pull_glob(h));
        std::memcpy(glob_no, h->glob_host.data(), sizeof(int32_t) * n);
    }
    return FM_OK;
}

extern "C" int fm_download_state_device(fm_handle *h, double *d_r, double *d_v, double *d_a)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (h->stage < 1) return fail(FM_ERR_STATE, "no state uploaded");
    fm::launch_gather_state(h->d, d_r, d_v, d_a, nullptr, nullptr, nullptr, h->st);
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

// ---------------------------------------------------------------------------
// device status
// ---------------------------------------------------------------------------

static int read_scalars(fm_handle *h, fm::FmScalars *s)
{
    FM_CUDA(cudaMemcpyAsync(s, h->d.sc, sizeof(*s), cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    return FM_OK;
}

static int status_error(fm_handle *h, const fm::FmScalars &s)
{
    char buf[256];
    if (s.status & fm::ST_ESCAPE) {
        std::snprintf(buf, sizeof buf, "molecule escaped the cell grid at iteration %d", s.fail_iter);
        h->stage = 3;
        return fail(FM_ERR_ESCAPE, buf);
    }
    if (s.status & fm::ST_PE) {
        std::snprintf(buf, sizeof buf, "max(potenergymol) > 10000 at iteration %d", s.fail_iter);
        h->stage = 3;
        return fail(FM_ERR_PE, buf);
    }
    if (s.status & fm::ST_BOND) {
        std::snprintf(buf, sizeof buf, "polymer bond beyond R_0 at iteration %d", s.fail_iter);
        h->stage = 3;
        return fail(FM_ERR_BOND, buf);
    }
    if (s.status & fm::ST_ANGLE) {
        std::snprintf(buf, sizeof buf,
                      "angular triple without a defined result (a middle bead without both bonds, or "
                      "k_ijk < 1e-5) at iteration %d", s.fail_iter);
        h->stage = 3;
        return fail(FM_ERR_BOND, buf);
    }
    if (s.status & fm::ST_TILE) {
        std::snprintf(buf, sizeof buf, "staged neighbourhood of %d molecules above the capacity %d at iteration %d",
                      s.umax, h->d.tile_ucap, s.fail_iter);
        h->stage = 3;
        return fail(FM_ERR_NLIST, buf);
    }
    if (s.status & fm::ST_MIGRATE) {
        std::snprintf(buf, sizeof buf,
                      "subdomain at iteration %d: a molecule moved beyond the neighbouring subdomains, or more "
                      "molecules arrived than the capacity holds", s.fail_iter);
        h->stage = 3;
        return fail(FM_ERR_ESCAPE, buf);
    }
    if (s.status & fm::ST_NLIST) {
        std::snprintf(buf, sizeof buf, "neighbour list overflow at iteration %d (%d > %d)", s.fail_iter, s.max_nbr,
                      h->d.tile ? h->d.maxn16 : h->d.maxn);
        h->stage = 3;
        return fail(FM_ERR_NLIST, buf);
    }
    return FM_OK;
}

// Status bits a larger capacity cures: the list (ST_NLIST) and, on the tiled
// path, the staged neighbourhood (ST_TILE).
static constexpr uint32_t GROWABLE = fm::ST_NLIST | fm::ST_TILE;
static bool growable(const fm::FmScalars &s)
{
    return (s.status & GROWABLE) && !(s.status & (fm::ST_FATAL & ~GROWABLE));
}

// Grows the neighbour list to fit the largest list seen (and, on the tiled
// path, the staging to fit the largest neighbourhood, leaving the tiled path
// when that no longer fits in shared memory), clears the overflow bits and
// rebuilds the list from the (frozen) current cells.
static int grow_nlist(fm_handle *h, const fm::FmScalars &s, int iter)
{
    FmDev &d = h->d;
    if (d.tile && (s.status & fm::ST_TILE)) {
        const int want_u = round_up((int)std::ceil(1.25 * s.umax) + 32, 32);
        if (want_u > fm::tile_ucap_limit(d.tile_R)) {
            FM_TRY(leave_tiles(h));
            d.nblocks_force = force_rows(h);
        } else {
            d.tile_ucap = want_u;
        }
    }
    if (s.status & fm::ST_NLIST) {
        const int cur = d.tile ? d.maxn16 : d.maxn;
        const int want = std::max(round_up((int)std::ceil(1.2 * s.max_nbr) + 8, 8), cur);
        if ((size_t)want * (size_t)d.n > ((size_t)1 << 34)) return status_error(h, s);
        FM_TRY(d.tile ? alloc_nlist16(h, want) : alloc_nlist(h, want));
    }
    fm::FmScalars t = s;
    t.status = 0u;
    t.fail_iter = -1;
    t.max_nbr = 0;
    FM_CUDA(cudaMemcpyAsync(d.sc, &t, sizeof t, cudaMemcpyHostToDevice, h->st));
    queue_build(h, 0, iter);
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

// ---------------------------------------------------------------------------
// pieces of the step
// ---------------------------------------------------------------------------

// sort_mols of a rebuild, after the periodic wrap and before the cell sort
// orders each cell's members by the (new) upload index.
static void queue_sort(fm_handle *h, int gated, cudaStream_t st)
{
    if (!h->sort_flag) return;
    fm::launch_sort(h->d, h->sdev, gated, st);
    h->launches += SORT_KERNELS;
}

static void queue_cells(fm_handle *h, int wrap, int gated)
{
    const FmDev &d = h->d;
    fm::launch_wrap_bin(d, wrap, 1, gated, h->iter, h->st);
    if (wrap) queue_sort(h, gated, h->st);
    fm::launch_scan_cells(d, gated, h->st);
    fm::launch_scatter(d, gated, h->st);
    fm::launch_reorder(d, gated, h->tpos, h->tuidx, h->st);
    h->launches += 7;
}

static cudaEvent_t next_event(fm_handle *h)
{
    if (h->ev_used == h->ev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        h->ev.push_back(e);
    }
    return h->ev[h->ev_used++];
}

static void queue_force(fm_handle *h, int record, int mode)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (h->timing) {
        e0 = next_event(h);
        e1 = next_event(h);
        if (e0) cudaEventRecord(e0, h->st);
    }
    if (h->p.force_list == 0) {
        FmDev d = h->d;
        d.nblocks_force = fm::all_pairs_blocks(d.n);
        fm::launch_all_pairs(d, record, mode, h->st);
    } else {
        fm::launch_force(h->d, record, mode, h->tpm, h->st);
    }
    if (e1) cudaEventRecord(e1, h->st);
    h->launches += 1;
}

// `pressure_sample`: simulation_record's pressure_averaging (:1189) runs with
// the record of a step; the setup record (setup_initial_record.f90:89) has none.
static void queue_record(fm_handle *h, int iter, double simtime, bool pressure_sample = true)
{
    FmDev d = h->d;
    if (!pressure_sample) d.pressure = 0;
    d.nblocks_force = h->p.force_list == 0 ? fm::all_pairs_blocks(d.n) : force_rows(h);
    fm::launch_record(d, iter, simtime, h->st);
    h->launches += 1;
}

// Threads-per-molecule autotuner: times the force kernel (forces only, no
// record) for TPM in {1, 2, 4, 8, 16} on the freshly built list and keeps the
// fastest.  The choice is cached per (np, expected neighbours, precision) for
// the process -- never per list capacity, which grows on overflow -- so handles
// created with equal parameters run identical kernels and give bit-identical
// results.
#include <map>
#include <mutex>
#include <tuple>
static std::mutex g_tune_mutex;
static std::map<std::tuple<int, int, int>, int> g_tune_cache;

static int autotune_tpm(fm_handle *h)
{
    // the tiled path's lanes per molecule are fixed by its row layout
    if (h->p.threads_per_molecule > 0 || h->p.force_list == 0 || h->d.tile) return FM_OK;
    const auto key = std::make_tuple(h->d.n, h->expected_nbr, h->d.precision);
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            h->tpm = it->second;
            h->d.nblocks_force = force_rows(h);
            return FM_OK;
        }
    }
    cudaEvent_t e0, e1;
    FM_CUDA(cudaEventCreate(&e0));
    FM_CUDA(cudaEventCreate(&e1));
    const int cands[5] = {1, 2, 4, 8, 16};
    float best = 1e30f;
    int best_tpm = h->tpm;
    float tbest[5] = {1e30f, 1e30f, 1e30f, 1e30f, 1e30f};
    for (int round = 0; round < 3; round++) {  // interleaved rounds, best of each candidate
        for (int c = 0; c < 5; c++) {
            const int t = cands[c];
            fm::launch_force(h->d, 0, 0, t, h->st);  // warm-up
            cudaEventRecord(e0, h->st);
            for (int rep = 0; rep < 2; rep++) fm::launch_force(h->d, 0, 0, t, h->st);
            cudaEventRecord(e1, h->st);
            cudaError_t err = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (err == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
            if (err == cudaSuccess && ms < tbest[c]) tbest[c] = ms;
        }
    }
    for (int c = 0; c < 5; c++)
        if (tbest[c] < best) { best = tbest[c]; best_tpm = cands[c]; }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    FM_CUDA(cudaGetLastError());
    h->tpm = best_tpm;
    h->d.nblocks_force = force_rows(h);
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tune_cache[key] = best_tpm;
    return FM_OK;
}

// Staged rows of the tiled path: w (Mie type, Soddemann bead flag) is staged
// when the potential reads it.
static void set_tile_rows(fm_handle *h)
{
    FmDev &d = h->d;
    if (!d.tile) return;
    d.tile_R = (d.mie || d.solvent) ? 4 : 3;
    if (d.tile_ucap > fm::tile_ucap_limit(d.tile_R)) d.tile_ucap = fm::tile_ucap_limit(d.tile_R);
}

extern "C" int fm_setup(fm_handle *h)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (h->d.dd) return fail(FM_ERR_STATE, "a subdomain handle is driven by the fm_dd_* calls");
    if (h->stage < 1) return fail(FM_ERR_STATE, "fm_setup before fm_upload_state");
    set_tile_rows(h);
    if (h->p.force_list != 0) {
        queue_cells(h, 0, 0);
        queue_build(h, 0, h->iter);
    }
    FM_CUDA(cudaGetLastError());
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    for (int attempt = 0; attempt < 4 && growable(s); attempt++) {
        FM_TRY(grow_nlist(h, s, h->iter));
        FM_TRY(read_scalars(h, &s));
    }
    FM_TRY(status_error(h, s));
    FM_TRY(autotune_tpm(h));
    const int record = (h->iter % h->p.tplot) == 0;
    queue_force(h, record, 0);
    if (record) queue_record(h, h->iter, h->simtime, false);
    FM_CUDA(cudaGetLastError());
    FM_TRY(read_scalars(h, &s));
    FM_TRY(status_error(h, s));
    h->has_pe = record;
    h->cells_valid = h->list_valid = h->p.force_list != 0;
    h->stage = 2;
    return FM_OK;
}

// Queues iterations [first, first + nsteps) of md_advance_vv, starting at
// `phase` 0 (move(1)) or 1 (forces) of the first iteration.
static void queue_decide(fm_handle *h, int it, int flip)
{
    const fm_params &p = h->p;
    if (p.rebuild_criteria == 2) { fm::launch_disp(h->d, h->st); h->launches += 1; }
    fm::launch_decide(h->d, it, flip, p.rebuild_criteria, p.fixed_rebuild, h->half_min_delta, h->st);
    h->launches += 1;
}

static void queue_rebuild_branch(fm_handle *h, int it, int flip);

static void queue_rebuild_check(fm_handle *h, int it, int flip)
{
    const fm_params &p = h->p;
    if (p.force_list != 0) {
        queue_rebuild_branch(h, it, flip);
    } else {
        queue_decide(h, it, flip);
        fm::launch_wrap_bin(h->d, 1, 0, 1, it, h->st);
        h->launches += 1;
        queue_sort(h, 1, h->st);
    }
}

// sort_mols inside the rebuild body being captured on h->cap_st2: the counter
// kernel, then a nested IF node that it sets on the rebuilds that sort, whose
// body (captured on h->cap_st3) holds the keys, the radix sort and the
// renumbering.  The other rebuilds skip the radix sort entirely.
static bool capture_sort(fm_handle *h)
{
    const FmDev &d = h->d;
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    if (!h->cap_st3 && cudaStreamCreateWithFlags(&h->cap_st3, cudaStreamNonBlocking) != cudaSuccess) return false;
    if (cudaStreamGetCaptureInfo(h->cap_st2, &cst, nullptr, &g, nullptr, nullptr) != cudaSuccess || !g) return false;
    cudaGraphConditionalHandle cond{};
    if (cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) return false;
    fm::launch_sort_gate_graph(d, h->sdev, cond, SORT_KERNELS - 1, h->cap_st2);
    if (cudaStreamGetCaptureInfo(h->cap_st2, &cst, nullptr, nullptr, &deps, &nd) != cudaSuccess) return false;
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t ifn = nullptr;
    if (cudaGraphAddNode(&ifn, g, deps, nd, &cp) != cudaSuccess) return false;
    if (cudaStreamUpdateCaptureDependencies(h->cap_st2, &ifn, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
        return false;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(h->cap_st3, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
        return false;
    fm::launch_sort_body(d, h->sdev, 1, h->cap_st3);
    return cudaStreamEndCapture(h->cap_st3, &body) == cudaSuccess;
}

// The rebuild branch of an iteration, appended to the graph being captured
// on h->cap_st: k_decide_graph (the iteration from the device counter g_iter)
// and an IF node whose body is the rebuild pipeline of queue_cells +
// queue_build, captured on h->cap_st2 with programmatic edges between its
// kernels as the stream launches have.
static bool capture_branch(fm_handle *h, int flip)
{
    const FmDev &d = h->d;
    const fm_params &p = h->p;
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    if (cudaStreamGetCaptureInfo(h->cap_st, &cst, nullptr, &g, nullptr, nullptr) != cudaSuccess || !g) return false;
    cudaGraphConditionalHandle cond{};
    if (cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) return false;
    const int body_kernels = 8 + (d.tile ? 1 : 0) + (d.angular ? 1 : 0) + (h->sort_flag ? 1 : 0);
    fm::launch_decide_graph(d, flip, p.rebuild_criteria, p.fixed_rebuild, h->half_min_delta, cond, body_kernels,
                            h->cap_st);
    if (cudaStreamGetCaptureInfo(h->cap_st, &cst, nullptr, nullptr, &deps, &nd) != cudaSuccess) return false;
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t ifn = nullptr;
    if (cudaGraphAddNode(&ifn, g, deps, nd, &cp) != cudaSuccess) return false;
    if (cudaStreamUpdateCaptureDependencies(h->cap_st, &ifn, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
        return false;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(h->cap_st2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
        return false;
    fm::pdl_capture = true;  // the body's first kernel has no predecessor to overlap
    fm::launch_wrap_bin(d, 1, 1, 1, fm::ITER_DEVICE, h->cap_st2);
    if (h->sort_flag && !capture_sort(h)) {
        cudaGraph_t body_again = nullptr;  // the node's own graph: ends the capture, nothing to free
        cudaStreamEndCapture(h->cap_st2, &body_again);
        return false;
    }
    fm::pdl_capture = h->sort_flag != 0;  // no programmatic edge out of the sort's conditional node
    fm::launch_scan_cells(d, 1, h->cap_st2);
    fm::pdl_capture = false;
    fm::launch_scatter(d, 1, h->cap_st2);
    fm::launch_reorder(d, 1, h->tpos, h->tuidx, h->cap_st2);
    if (d.tile) fm::launch_blk_seg(d, 1, fm::ITER_DEVICE, h->cap_st2);
    fm::launch_build_nlist(d, 1, fm::ITER_DEVICE, h->cap_st2);
    if (d.angular) fm::launch_angular_order(d, 1, fm::ITER_DEVICE, h->cap_st2);
    fm::pdl_capture = true;
    return cudaStreamEndCapture(h->cap_st2, &body) == cudaSuccess;
}

// Iterations per graph launch in the middle of a range.
constexpr int STEP_GRAPH_K = 8;

// No iteration of [it, it + k) is a record step.
static bool no_record_in(int it, int k, int tplot)
{
    for (int j = 0; j < k; j++)
        if (((it + j) % tplot) == 0) return false;
    return true;
}

// Graph of `k` iterations (k = 0: the rebuild branch of one iteration only):
// per iteration the rebuild branch and, for k > 0, the non-recording force
// kernel with move(2) and the next move(1) (mode 2), as queue_steps launches
// them for an iteration in the middle of a range.  The first branch takes
// `flip`, the later ones 1 (move(1) was fused into the force kernel before
// them).  Cached per (flip, k) until the device state it was captured with
// (FmDev) or the lanes per molecule change; null where graphs cannot be made.
static cudaGraphExec_t step_graph(fm_handle *h, int flip, int k)
{
    if (h->rb_off) return nullptr;
    const int slot = 2 * (k > 0) + flip;
    if (h->rbx[slot] && h->rbt[slot] == h->tpm && std::memcmp(&h->rbd[slot], &h->d, sizeof(FmDev)) == 0)
        return h->rbx[slot];
    if (h->rbx[slot]) { cudaGraphExecDestroy(h->rbx[slot]); h->rbx[slot] = nullptr; }
    bool ok = (h->cap_st || cudaStreamCreateWithFlags(&h->cap_st, cudaStreamNonBlocking) == cudaSuccess) &&
              (h->cap_st2 || cudaStreamCreateWithFlags(&h->cap_st2, cudaStreamNonBlocking) == cudaSuccess);
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    fm::pdl_capture = true;
    if (ok && cudaStreamBeginCapture(h->cap_st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        for (int s = 0; ok && s < std::max(k, 1); s++) {
            ok = capture_branch(h, s == 0 ? flip : 1);
            if (ok && k > 0) fm::launch_force(h->d, 0, 2, h->tpm, h->cap_st);
        }
        cudaGraph_t got = nullptr;
        const bool ended = cudaStreamEndCapture(h->cap_st, &got) == cudaSuccess;
        g = got;
        ok = ok && ended && g;
    } else {
        ok = false;
    }
    fm::pdl_capture = false;
    if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
        if (ex) cudaGraphExecDestroy(ex);
        cudaGetLastError();  // the per-kernel path takes over
        h->rb_off = true;
        return nullptr;
    }
    h->rbx[slot] = ex;
    h->rbd[slot] = h->d;
    h->rbt[slot] = h->tpm;
    return ex;
}

// The rebuild check of iteration `it` on the cell path: the graph when there
// is one (g_iter set by the caller at the start of its range), else the
// decision and the gated rebuild kernels one launch each.
static void queue_rebuild_branch(fm_handle *h, int it, int flip)
{
    const fm_params &p = h->p;
    cudaGraphExec_t ex = step_graph(h, flip, 0);
    if (ex) {
        if (p.rebuild_criteria == 2) { fm::launch_disp(h->d, h->st); h->launches += 1; }
        cudaGraphLaunch(ex, h->st);
        h->launches += 1;  // the decision; the body's kernels are counted on the device
        return;
    }
    queue_decide(h, it, flip);
    queue_cells(h, 1, 1);
    queue_build(h, 1, it);
    h->launches += 1;
}

// Leap-frog iterations [first, first + nsteps): forces + record + move fused,
// then the rebuild check and gated rebuild of the same iteration.
static int queue_steps_lfv(fm_handle *h, int first, int nsteps, const std::vector<double> &simtime_after,
                           int range_offset)
{
    if (h->p.force_list != 0 && nsteps > 0) fm::launch_set_graph_iter(h->d, first, h->st);
    for (int s = 0; s < nsteps; s++) {
        const int it = first + s;
        h->iter = it;
        const int record = (it % h->p.tplot) == 0;
        const double t_before = h->simtime;
        queue_force(h, record, 3);
        if (record) queue_record(h, it, t_before);
        h->simtime = simtime_after[(size_t)(range_offset + s)];
        queue_rebuild_check(h, it, 1);
    }
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

static int queue_steps(fm_handle *h, int first, int nsteps, int phase, const std::vector<double> &simtime_after,
                       int range_offset)
{
    const fm_params &p = h->p;
    if (p.integration_algorithm == 0) return queue_steps_lfv(h, first, nsteps, simtime_after, range_offset);
    bool fused_move1 = false;  // the previous force kernel already did move(1)
    if (p.force_list != 0 && nsteps > (phase == 1 ? 1 : 0))  // the first decision's iteration
        fm::launch_set_graph_iter(h->d, phase == 1 ? first + 1 : first, h->st);
    for (int s = 0; s < nsteps; s++) {
        const int it = first + s;
        h->iter = it;
        // STEP_GRAPH_K middle iterations in one graph launch: none records,
        // none is the range's last, move(1) of the first is already done
        if (fused_move1 && p.force_list != 0 && p.rebuild_criteria != 2 && !h->timing && s + STEP_GRAPH_K < nsteps &&
            no_record_in(it, STEP_GRAPH_K, p.tplot)) {
            cudaGraphExec_t ex = step_graph(h, 1, STEP_GRAPH_K);
            if (ex) {
                cudaGraphLaunch(ex, h->st);
                h->launches += 2 * STEP_GRAPH_K;  // decisions and force kernels
                s += STEP_GRAPH_K - 1;
                h->iter = first + s;
                h->simtime = simtime_after[(size_t)(range_offset + s)];
                continue;
            }
        }
        if (!(s == 0 && phase == 1)) {
            if (!fused_move1) { fm::launch_move1(h->d, h->st); h->launches += 1; }
            if (p.force_list != 0) {
                queue_rebuild_branch(h, it, fused_move1 ? 1 : 0);
            } else {
                queue_decide(h, it, fused_move1 ? 1 : 0);
                fm::launch_wrap_bin(h->d, 1, 0, 1, it, h->st);
                h->launches += 1;
                queue_sort(h, 1, h->st);
            }
        }
        const int record = (it % p.tplot) == 0;
        const int last = s == nsteps - 1;
        queue_force(h, record, last ? 1 : 2);
        fused_move1 = !last;
        h->simtime = simtime_after[(size_t)(range_offset + s)];
        if (record) queue_record(h, it, h->simtime);
    }
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

// Waits for the queued range; resumes it once per overflow after growing the
// neighbour list.
static int finish_range(fm_handle *h)
{
    for (int attempt = 0; attempt < 8; attempt++) {
        fm::FmScalars s;
        FM_TRY(read_scalars(h, &s));
        if (!(s.status & fm::ST_FATAL)) {
            h->q.active = false;
            return FM_OK;
        }
        if (!h->q.active || (s.status & (fm::ST_FATAL & ~GROWABLE))) {
            h->q.active = false;
            return status_error(h, s);
        }
        const int f = s.fail_iter;
        const int off = f - h->q.first_iter;
        if (off < 0 || off >= h->q.nsteps) return status_error(h, s);
        FM_TRY(grow_nlist(h, s, f));
        if (h->p.integration_algorithm == 0) {
            // the list of iteration f overflowed after its move: go on with f + 1
            h->simtime = h->q.simtime_after[(size_t)off];
            FM_TRY(queue_steps(h, f + 1, h->q.nsteps - off - 1, 0, h->q.simtime_after, off + 1));
        } else {
            FM_TRY(queue_steps(h, f, h->q.nsteps - off, 1, h->q.simtime_after, off));
        }
    }
    return fail(FM_ERR_NLIST, "neighbour list kept overflowing");
}

extern "C" int fm_step(fm_handle *h, int32_t nsteps, int32_t blocking)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (h->d.dd) return fail(FM_ERR_STATE, "a subdomain handle is driven by the fm_dd_* calls");
    if (h->stage != 2) return fail(FM_ERR_STATE, "fm_step needs fm_setup (or a failed state was not re-uploaded)");
    if (h->p.force_list != 0 && !(h->cells_valid && h->list_valid))
        return fail(FM_ERR_STATE, "fm_step needs current cell and neighbour lists (call fm_setup)");
    if (nsteps < 0) return fail(FM_ERR_ARG, "nsteps < 0");
    if (nsteps == 0) return FM_OK;
    if (h->q.active) FM_TRY(finish_range(h));
    const int first = h->iter + 1;
    h->q.active = true;
    h->q.first_iter = first;
    h->q.nsteps = nsteps;
    h->q.simtime_after.resize((size_t)nsteps);
    double t = h->simtime;
    for (int s = 0; s < nsteps; s++) {
        t = t + h->p.delta_t;  // simtime = simtime + delta_t (simulation_move_particles_vv.f90:191)
        h->q.simtime_after[(size_t)s] = t;
    }
    FM_TRY(queue_steps(h, first, nsteps, 0, h->q.simtime_after, 0));
    for (int s = 0; s < nsteps; s++)
        if (((first + s) % h->p.tplot) == 0) h->has_pe = true;
    if (blocking) return finish_range(h);
    return FM_OK;
}

extern "C" int fm_sync(fm_handle *h)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (h->q.active) return finish_range(h);
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    return status_error(h, s);
}

// ---------------------------------------------------------------------------
// subroutine-by-subroutine mirrors
// ---------------------------------------------------------------------------

static int ready(fm_handle *h, int min_stage)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (h->d.dd) return fail(FM_ERR_STATE, "a subdomain handle is driven by the fm_dd_* calls");
    if (h->stage == 3) return fail(FM_ERR_STATE, "state is broken; re-upload it");
    if (h->stage < min_stage) return fail(FM_ERR_STATE, "call order: upload, setup, then step");
    if (h->q.active) FM_TRY(finish_range(h));
    return FM_OK;
}

extern "C" int fm_move_vv(fm_handle *h, int32_t pass_num)
{
    FM_TRY(ready(h, 1));
    if (pass_num == 1) {
        fm::launch_move1(h->d, h->st);
    } else if (pass_num == 2) {
        fm::launch_move2(h->d, h->st);
        h->simtime = h->simtime + h->p.delta_t;
    } else {
        return fail(FM_ERR_ARG, "pass_num must be 1 or 2");
    }
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

extern "C" int fm_move_lfv(fm_handle *h)
{
    FM_TRY(ready(h, 1));
    fm::launch_move_lfv(h->d, h->st);
    h->simtime = h->simtime + h->p.delta_t;
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

extern "C" int fm_update_borders(fm_handle *h, int32_t rebuild)
{
    (void)rebuild;
    return ready(h, 1);
}

extern "C" int fm_linklist_deallocateall(fm_handle *h) { return ready(h, 1); }

extern "C" int fm_check_rebuild(fm_handle *h, int32_t *rebuild)
{
    FM_TRY(ready(h, 1));
    if (!rebuild) return fail(FM_ERR_ARG, "null output");
    FM_CUDA(cudaMemsetAsync(&h->d.sc->vmax2, 0, sizeof(unsigned long long), h->st));
    fm::launch_vmax(h->d, h->st);
    queue_decide(h, h->iter, 0);
    FM_CUDA(cudaGetLastError());
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    FM_TRY(status_error(h, s));
    *rebuild = s.rebuild;
    return FM_OK;
}

extern "C" int fm_set_sort(fm_handle *h, int32_t sort_flag, int32_t sort_freq, int32_t sortblocksize)
{
    FM_TRY(ready(h, 1));  // refuses a subdomain handle: its molecules are named by global number
    if (sort_flag < 0 || sort_flag > 2) return fail(FM_ERR_ARG, "Incorrect value of sort_flag");
    if (sort_flag != 0 && h->p.potential_flag == 1)
        return fail(FM_ERR_ARG, "Sort should be turned off - Not developed for polymers");
    if (sort_flag != 0 && h->d.mie) return fail(FM_ERR_ARG, "Sort should be turned off - Not developed for Mie potential");
    if (sort_flag != 0 && sortblocksize < 1) return fail(FM_ERR_ARG, "sortblocksize must be at least 1");
    FM_TRY(fm_sync(h));
    release_graphs(h);  // recaptured with or without the sort kernels
    free_sort(h);
    if (sort_flag == 0) return FM_OK;
    fm::FmSortDev s{};
    long long blocks = 1;
    for (int k = 0; k < 3; k++) {
        s.bsl[k] = (double)sortblocksize * h->d.cs[k];  // blocksidelength (linklist.f90:2790-2791)
        s.nb[k] = (int)std::ceil(h->d.L[k] / s.bsl[k]);
        blocks *= s.nb[k];
    }
    if (blocks > (1ll << 26)) return fail(FM_ERR_ARG, "sort blocks: more than 2^26");
    std::vector<int32_t> hc((size_t)blocks);
    const char *why = nullptr;
    if (fm::sort_table(sort_flag, s.nb, hc.data(), &why) != 0) return fail(FM_ERR_ARG, why);
    s.freq = sort_freq;
    s.blocks = (int)blocks;
    s.end_bit = 1;
    while ((1ll << s.end_bit) < blocks) s.end_bit++;
    const int n = h->d.n;
    int32_t *hcd = nullptr;
    std::vector<int32_t> iota((size_t)n);
    for (int i = 0; i < n; i++) iota[(size_t)i] = i;
    fm::FmSortScalars q{};
    q.nrebuilds = 1;
    q.sf1 = 1.5;
    q.sf2 = 5;
    s.tmp_bytes = fm::sort_scratch_bytes(n, s.end_bit);
    h->sdev = s;  // free_sort releases whatever the allocations below got
    fm::FmSortDev &t = h->sdev;
    FM_TRY(dalloc(&hcd, (size_t)blocks));
    t.hc = hcd;
    FM_TRY(dalloc(&t.key, n)); FM_TRY(dalloc(&t.key_out, n)); FM_TRY(dalloc(&t.val, n));
    FM_TRY(dalloc(&t.val_out, n)); FM_TRY(dalloc(&t.cnt, (size_t)blocks)); FM_TRY(dalloc(&t.newv, n));
    FM_TRY(dalloc(&t.gtmp, n)); FM_TRY(dalloc(&t.ss, 1));
    FM_CUDA(cudaMalloc(&t.tmp, std::max<size_t>(t.tmp_bytes, 16)));
    t.glob = h->glob;
    FM_CUDA(cudaMemcpyAsync(hcd, hc.data(), sizeof(int32_t) * (size_t)blocks, cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaMemcpyAsync(t.val, iota.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaMemsetAsync(t.key, 0, sizeof(int32_t) * (size_t)n, h->st));
    FM_CUDA(cudaMemsetAsync(t.cnt, 0, sizeof(int32_t) * (size_t)blocks, h->st));
    FM_CUDA(cudaMemcpyAsync(t.ss, &q, sizeof(q), cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));  // the host vectors go out of scope
    h->sort_flag = sort_flag;
    h->glob_moved = true;
    return FM_OK;
}

extern "C" int fm_get_sort_state(fm_handle *h, int64_t *sorts, int64_t *skipped, int32_t *nrebuilds, double *sf1,
                                 int32_t *sf2)
{
    FM_TRY(ready(h, 1));
    fm::FmSortScalars q{};
    q.nrebuilds = 1;
    q.sf1 = 1.5;
    q.sf2 = 5;
    if (h->sort_flag) {
        FM_CUDA(cudaMemcpyAsync(&q, h->sdev.ss, sizeof(q), cudaMemcpyDeviceToHost, h->st));
        FM_CUDA(cudaStreamSynchronize(h->st));
    }
    if (sorts) *sorts = q.sorts;
    if (skipped) *skipped = q.skipped;
    if (nrebuilds) *nrebuilds = q.nrebuilds;
    if (sf1) *sf1 = q.sf1;
    if (sf2) *sf2 = q.sf2;
    return FM_OK;
}

extern "C" int fm_sort_mols(fm_handle *h)
{
    FM_TRY(ready(h, 1));
    queue_sort(h, 0, h->st);
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

extern "C" int fm_sendmols(fm_handle *h)
{
    FM_TRY(ready(h, 1));
    fm::launch_wrap_bin(h->d, 1, 0, 0, h->iter, h->st);
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

extern "C" int fm_assign_to_cell(fm_handle *h)
{
    FM_TRY(ready(h, 1));
    if (h->p.force_list == 0) return FM_OK;
    queue_cells(h, 0, 0);
    FM_CUDA(cudaGetLastError());
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    FM_TRY(status_error(h, s));
    h->cells_valid = true;
    h->list_valid = false;
    return FM_OK;
}

extern "C" int fm_assign_to_neighbourlist(fm_handle *h)
{
    FM_TRY(ready(h, 1));
    if (h->p.force_list == 0) return FM_OK;
    if (!h->cells_valid) return fail(FM_ERR_STATE, "assign_to_neighbourlist needs assign_to_cell first");
    set_tile_rows(h);
    queue_build(h, 0, h->iter);
    FM_CUDA(cudaGetLastError());
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    for (int attempt = 0; attempt < 4 && growable(s); attempt++) {
        FM_TRY(grow_nlist(h, s, h->iter));
        FM_TRY(read_scalars(h, &s));
    }
    FM_TRY(status_error(h, s));
    h->list_valid = true;
    return FM_OK;
}

// The rebuild branch of md_advance_vv (md.f90:150-157) in one call.
extern "C" int fm_rebuild_lists(fm_handle *h)
{
    FM_TRY(fm_linklist_deallocateall(h));
    FM_TRY(fm_sendmols(h));
    FM_TRY(fm_sort_mols(h));
    FM_TRY(fm_assign_to_cell(h));
    FM_TRY(fm_update_borders(h, 1));
    return fm_assign_to_neighbourlist(h);
}

extern "C" int fm_compute_forces(fm_handle *h)
{
    FM_TRY(ready(h, 1));
    if (h->p.force_list != 0 && !(h->cells_valid && h->list_valid))
        return fail(FM_ERR_STATE, "compute_forces needs assign_to_cell and assign_to_neighbourlist first");
    const int record = (h->iter % h->p.tplot) == 0;
    queue_force(h, record, 0);
    FM_CUDA(cudaGetLastError());
    if (record) h->has_pe = true;
    if (h->stage < 2) h->stage = 2;
    return FM_OK;
}

extern "C" int fm_evaluate_macroscopic_properties(fm_handle *h, fm_macro *out)
{
    FM_TRY(ready(h, 2));
    if (!out) return fail(FM_ERR_ARG, "null output");
    FmDev d = h->d;
    d.nblocks_force = fm::macro_blocks(d.n);
    fm::launch_macro_partials(d, h->st);
    fm::launch_record(d, h->iter, h->simtime, h->st);
    FM_CUDA(cudaGetLastError());
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    FM_TRY(status_error(h, s));
    int slot = (s.nrec_pending - 1 + d.rec_cap) % d.rec_cap;
    static_assert(sizeof(fm::FmRecord) == sizeof(fm_macro), "record layout");
    FM_CUDA(cudaMemcpyAsync(out, d.rec + slot, sizeof(fm_macro), cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    return FM_OK;
}

extern "C" int fm_set_iter(fm_handle *h, int32_t iter)
{
    FM_TRY(ready(h, 0));
    h->iter = iter;
    return FM_OK;
}

extern "C" int fm_get_iter(fm_handle *h, int32_t *iter)
{
    if (!h || !iter) return fail(FM_ERR_ARG, "null argument");
    *iter = h->iter;
    return FM_OK;
}

// ---------------------------------------------------------------------------
// results
// ---------------------------------------------------------------------------

extern "C" int fm_get_records(fm_handle *h, fm_macro *out, int32_t cap, int32_t *n)
{
    if (!h || !n) return fail(FM_ERR_ARG, "null argument");
    if (h->q.active) FM_TRY(finish_range(h));
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    const int rc_cap = h->d.rec_cap;
    int pending = s.nrec_pending;
    int avail = std::min(pending, rc_cap);
    int take = std::min(avail, cap > 0 ? cap : 0);
    std::vector<fm::FmRecord> rows((size_t)rc_cap);
    if (take > 0) {
        FM_CUDA(cudaMemcpyAsync(rows.data(), h->d.rec, sizeof(fm::FmRecord) * (size_t)rc_cap, cudaMemcpyDeviceToHost,
                                h->st));
        FM_CUDA(cudaStreamSynchronize(h->st));
        int oldest = pending - avail;
        for (int k = 0; k < take; k++) std::memcpy(&out[k], &rows[(size_t)((oldest + k) % rc_cap)], sizeof(fm_macro));
    }
    int zero = 0;
    FM_CUDA(cudaMemcpyAsync(&h->d.sc->nrec_pending, &zero, sizeof zero, cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    *n = take;
    return FM_OK;
}

extern "C" int fm_get_per_molecule(fm_handle *h, double *pe, double *vir)
{
    FM_TRY(ready(h, 2));
    const size_t n = (size_t)h->d.n;
    double *dpe = h->stage3, *dvir = h->stage3 + n;
    fm::launch_gather_state(h->d, nullptr, nullptr, nullptr, nullptr, dpe, dvir, h->st);
    if (pe) FM_CUDA(cudaMemcpyAsync(pe, dpe, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
    if (vir) FM_CUDA(cudaMemcpyAsync(vir, dvir, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    return FM_OK;
}

// The current rows in the generic int32 layout: the list itself, or on the
// tiled path a temporary decoded copy (the caller frees it when it differs
// from d.nbr).  Test hooks only.
static int generic_rows(fm_handle *h, int32_t **out, int *maxn)
{
    if (!h->d.tile) { *out = h->d.nbr; *maxn = h->d.maxn; return FM_OK; }
    int32_t *buf = nullptr;
    FM_TRY(dalloc(&buf, fm::nb_rows(h->d.n) * (size_t)h->d.maxn16));
    fm::launch_tile_to_generic(h->d, buf, h->d.maxn16, h->st);
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) { cudaFree(buf); FM_CUDA(ce); }
    *out = buf;
    *maxn = h->d.maxn16;
    return FM_OK;
}

extern "C" int fm_get_pair_list(fm_handle *h, int32_t *owner, int32_t *partner, int8_t *code, int64_t cap,
                                int64_t *n_out)
{
    FM_TRY(ready(h, 1));
    if (!n_out) return fail(FM_ERR_ARG, "null output");
    if (h->p.force_list == 0) { *n_out = 0; return FM_OK; }
    const size_t n = (size_t)h->d.n;
    int32_t *dnbr = nullptr;
    int maxn = 0;
    FM_TRY(generic_rows(h, &dnbr, &maxn));
    std::vector<int32_t> nnbr(n), slot(n), nbr(fm::nb_rows((int)n) * (size_t)maxn);
    FM_CUDA(cudaMemcpyAsync(nnbr.data(), h->d.nnbr, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaMemcpyAsync(slot.data(), h->d.slot_of, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, h->st));
    cudaError_t ce = cudaMemcpyAsync(nbr.data(), dnbr, sizeof(int32_t) * nbr.size(), cudaMemcpyDeviceToHost, h->st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->st);
    if (dnbr != h->d.nbr) cudaFree(dnbr);
    FM_CUDA(ce);
    FM_TRY(pull_glob(h));
    int64_t k = 0;
    for (size_t i = 0; i < n; i++) {
        for (int q = 0; q < nnbr[i]; q++) {
            int32_t e = nbr[fm::nb_row((int)i, maxn) + fm::nb_col(q)];
            int32_t j = e & fm::NB_INDEX_MASK;
            int c6 = (int)((uint32_t)e >> fm::NB_SHIFT_BITS);
            int sx = (c6 & 3) - 1, sy = ((c6 >> 2) & 3) - 1, sz = ((c6 >> 4) & 3) - 1;
            if (k < cap) {
                if (owner) owner[k] = h->glob_host[(size_t)slot[i]];
                if (partner) partner[k] = h->glob_host[(size_t)slot[(size_t)j]];
                if (code) code[k] = (int8_t)((sx + 1) + 3 * (sy + 1) + 9 * (sz + 1));
            }
            k++;
        }
    }
    *n_out = k;
    return FM_OK;
}

extern "C" int fm_pair_digest(fm_handle *h, uint64_t *digest, int64_t *npairs)
{
    FM_TRY(ready(h, 1));
    if (!digest || !npairs) return fail(FM_ERR_ARG, "null output");
    if (h->p.force_list == 0) { *digest = 0; *npairs = 0; return FM_OK; }
    int32_t *dnbr = nullptr;
    int maxn = 0;
    FM_TRY(generic_rows(h, &dnbr, &maxn));
    FmDev d = h->d;
    d.nbr = dnbr;
    d.maxn = maxn;
    FM_CUDA(cudaMemsetAsync(&h->d.sc->digest, 0, sizeof(uint64_t) + sizeof(int64_t), h->st));
    fm::launch_pair_digest(d, h->glob, h->st);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->st);
    if (dnbr != h->d.nbr) cudaFree(dnbr);
    FM_CUDA(ce);
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    *digest = s.digest;
    *npairs = s.digest_n;
    return FM_OK;
}

extern "C" int fm_get_threads_per_molecule(fm_handle *h, int32_t *tpm)
{
    if (!h || !tpm) return fail(FM_ERR_ARG, "null argument");
    *tpm = h->tpm;
    return FM_OK;
}

extern "C" int fm_get_force_path(fm_handle *h, int32_t *path, int32_t *tile_capacity)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (path) *path = h->d.tile ? FM_FORCE_PATH_TILES : FM_FORCE_PATH_GATHER;
    if (tile_capacity) *tile_capacity = h->d.tile ? h->d.tile_ucap : 0;
    return FM_OK;
}

extern "C" int fm_get_counters(fm_handle *h, int64_t *rebuilds, int32_t *cap, int32_t *max_nbr)
{
    FM_TRY(ready(h, 0));
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    if (rebuilds) *rebuilds = s.rebuilds;
    if (cap) *cap = h->d.tile ? h->d.maxn16 : h->d.maxn;
    if (max_nbr) *max_nbr = s.max_nbr;
    return FM_OK;
}

extern "C" int fm_set_pressure_outflag(fm_handle *h, int32_t flag)
{
    FM_TRY(ready(h, 1));
    if (flag != 0 && flag != 1)
        return fail(FM_ERR_ARG, "pressure_outflag must be 0 or 1 (the volume-averaged forms are not built)");
    FmDev &d = h->d;
    if (flag == 1 && !d.rf6) {
        double *p = nullptr;
        FM_CUDA(cudaMalloc(&p, sizeof(double) * 6 * (size_t)d.n));
        d.rf6 = p;
        FM_CUDA(cudaMemsetAsync(d.rf6, 0, sizeof(double) * 6 * (size_t)d.n, h->st));
    }
    d.pressure = flag;
    FM_CUDA(cudaMemsetAsync(d.sc->pacc, 0, sizeof(d.sc->pacc), h->st));
    FM_CUDA(cudaMemsetAsync(&d.sc->pcount, 0, sizeof(int32_t), h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    return FM_OK;
}

extern "C" int fm_get_pressure_tensor(fm_handle *h, double P[9], int32_t *nsamples, int32_t reset)
{
    FM_TRY(ready(h, 1));
    if (!P) return fail(FM_ERR_ARG, "null output");
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    const int n = s.pcount;
    const double *a = s.pacc;  // xx yy zz xy xz yz
    const double m[9] = {a[0], a[3], a[4], a[3], a[1], a[5], a[4], a[5], a[2]};
    for (int q = 0; q < 9; q++) P[q] = n > 0 ? m[q] / (double)n : 0.0;
    if (nsamples) *nsamples = n;
    if (reset) {
        FM_CUDA(cudaMemsetAsync(h->d.sc->pacc, 0, sizeof(s.pacc), h->st));
        FM_CUDA(cudaMemsetAsync(&h->d.sc->pcount, 0, sizeof(int32_t), h->st));
        FM_CUDA(cudaStreamSynchronize(h->st));
    }
    return FM_OK;
}

// ---------------------------------------------------------------------------
// instrumentation
// ---------------------------------------------------------------------------

extern "C" int fm_force_kernel_timing(fm_handle *h, int32_t enable)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    h->timing = enable != 0;
    h->ev_used = 0;
    return FM_OK;
}

extern "C" int fm_get_force_kernel_time(fm_handle *h, double *ms, int64_t *launches)
{
    if (!h || !ms || !launches) return fail(FM_ERR_ARG, "null argument");
    FM_CUDA(cudaStreamSynchronize(h->st));
    double tot = 0.0;
    for (size_t k = 0; k + 1 < h->ev_used; k += 2) {
        float t = 0.f;
        FM_CUDA(cudaEventElapsedTime(&t, h->ev[k], h->ev[k + 1]));
        tot += (double)t;
    }
    *ms = tot;
    *launches = (int64_t)(h->ev_used / 2);
    h->ev_used = 0;
    return FM_OK;
}

extern "C" int fm_get_launch_count(fm_handle *h, int64_t *launches)
{
    if (!h || !launches) return fail(FM_ERR_ARG, "null argument");
    int64_t body = 0;  // kernels run inside the rebuild graph's conditional body
    if (h->d.sc) {
        fm::FmScalars s;
        FM_TRY(read_scalars(h, &s));
        body = s.graph_kernels;
    }
    *launches = h->launches + body;
    return FM_OK;
}

// ---------------------------------------------------------------------------
// spatial decomposition: one rank's subdomain (messenger.MPI.f90)
//
// The caller (one process per GPU, or several subdomains in one process)
// runs the exchanges between the calls: counts and flat record buffers in
// device memory, rank to rank (an all-to-all).  A rebuild is
//   fm_dd_classify -> exchange counts -> fm_dd_pack_emigrants -> exchange
//   -> fm_dd_immigrate -> fm_dd_halo_counts -> exchange counts
//   -> fm_dd_pack_halo -> exchange -> fm_dd_receive_halo (sort + list build);
// a step without a rebuild refreshes the halo positions
// (fm_dd_gather_positions -> exchange -> fm_dd_scatter_positions).
// ---------------------------------------------------------------------------

extern "C" int fm_dd_create(const fm_params *p, const int32_t ncells_global[3], const int32_t origin[3],
                            const int32_t ncells_local[3], int32_t capacity, fm_handle **out)
{
    if (!ncells_global || !origin || !ncells_local) return fail(FM_ERR_ARG, "null argument");
    DdGeom g;
    for (int k = 0; k < 3; k++) { g.nglob[k] = ncells_global[k]; g.org[k] = origin[k]; g.nloc[k] = ncells_local[k]; }
    g.capacity = capacity;
    return create_impl(p, &g, out);
}

static int dd_ready(fm_handle *h, bool planned, int min_stage)
{
    if (!h) return fail(FM_ERR_ARG, "null handle");
    if (!h->d.dd) return fail(FM_ERR_STATE, "not a subdomain handle (fm_dd_create)");
    if (planned && !h->planned) return fail(FM_ERR_STATE, "fm_dd_set_plan first");
    if (h->stage == 3) return fail(FM_ERR_STATE, "state is broken; re-upload it");
    if (h->stage < min_stage) return fail(FM_ERR_STATE, "call order: fm_dd_upload, a rebuild, then forces");
    return FM_OK;
}

extern "C" int fm_dd_set_plan(fm_handle *h, int32_t rank, const int32_t dims[3], const int32_t *owner_axis,
                              const int32_t *need_off, const int32_t *need_rank, const int32_t *need_code,
                              const int32_t *need_cell)
{
    FM_TRY(dd_ready(h, false, 0));
    if (!dims || !owner_axis || !need_off) return fail(FM_ERR_ARG, "null argument");
    const FmDev &d = h->d;
    const int nranks = dims[0] * dims[1] * dims[2];
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || rank < 0 || rank >= nranks)
        return fail(FM_ERR_ARG, "rank outside the process grid");
    const int G = (d.gne[0] - 2) + (d.gne[1] - 2) + (d.gne[2] - 2);
    const int nc = d.ncell;
    for (int k = 0; k < G; k++) {
        const int ax = k < d.gne[0] - 2 ? 0 : (k < d.gne[0] - 2 + d.gne[1] - 2 ? 1 : 2);
        if (owner_axis[k] < 0 || owner_axis[k] >= dims[ax]) return fail(FM_ERR_ARG, "owner_axis out of range");
    }
    if (need_off[0] != 0) return fail(FM_ERR_ARG, "need_off[0] must be 0");
    for (int c = 0; c < nc; c++)
        if (need_off[c + 1] < need_off[c]) return fail(FM_ERR_ARG, "need_off must be non-decreasing");
    const int nneed = need_off[nc];
    if (nneed > 0 && (!need_rank || !need_code || !need_cell)) return fail(FM_ERR_ARG, "null argument");
    for (int k = 0; k < nneed; k++)
        if (need_rank[k] < 0 || need_rank[k] >= nranks || need_code[k] < 0 || need_code[k] > 63 ||
            need_cell[k] < 0)
            return fail(FM_ERR_ARG, "need entries out of range");
    // one device block: owner_axis | need_off | need_rank | need_code | need_cell
    //                   | count | offset | cursor | nlist | list_idx | list_aux
    const size_t total = (size_t)G + (size_t)nc + 1 + 3 * (size_t)nneed + 3 * (size_t)nranks + 1 + 2 * (size_t)h->cap;
    if (h->dd_dev) cudaFree(h->dd_dev);
    h->dd_dev = nullptr;
    FM_TRY(dalloc(&h->dd_dev, total));
    if (!h->dd_sums) FM_TRY(dalloc(&h->dd_sums, (size_t)fm::RS_N));
    int32_t *b = h->dd_dev;
    fm::DdDev &x = h->x;
    x.rank = rank;
    for (int k = 0; k < 3; k++) x.dims[k] = dims[k];
    x.owner_axis = b; b += G;
    x.need_off = b; b += nc + 1;
    x.need_rank = b; b += nneed;
    x.need_code = b; b += nneed;
    x.need_cell = b; b += nneed;
    x.count = b; b += nranks;
    x.offset = b; b += nranks;
    x.cursor = b; b += nranks;
    x.nlist = b; b += 1;
    x.list_idx = b; b += h->cap;
    x.list_aux = b; b += h->cap;
    x.list_cap = h->cap;
    FM_CUDA(cudaMemcpyAsync((void *)x.owner_axis, owner_axis, sizeof(int32_t) * G, cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaMemcpyAsync((void *)x.need_off, need_off, sizeof(int32_t) * (nc + 1), cudaMemcpyHostToDevice, h->st));
    if (nneed > 0) {
        FM_CUDA(cudaMemcpyAsync((void *)x.need_rank, need_rank, sizeof(int32_t) * nneed, cudaMemcpyHostToDevice, h->st));
        FM_CUDA(cudaMemcpyAsync((void *)x.need_code, need_code, sizeof(int32_t) * nneed, cudaMemcpyHostToDevice, h->st));
        FM_CUDA(cudaMemcpyAsync((void *)x.need_cell, need_cell, sizeof(int32_t) * nneed, cudaMemcpyHostToDevice, h->st));
    }
    FM_CUDA(cudaStreamSynchronize(h->st));
    h->nranks = nranks;
    h->dd_counts.assign((size_t)nranks, 0);
    h->planned = true;
    return FM_OK;
}

extern "C" int fm_dd_upload(fm_handle *h, int32_t n, const double *r, const double *v, const int32_t *gid)
{
    FM_TRY(dd_ready(h, false, 0));
    if (n < 0 || n > h->cap) return fail(FM_ERR_ARG, "n outside 0 .. capacity");
    if (n > 0 && (!r || !v || !gid)) return fail(FM_ERR_ARG, "null argument");
    for (int i = 0; i < n; i++)
        if (gid[i] < 0 || gid[i] >= fm::MAX_MOLECULES) return fail(FM_ERR_ARG, "global numbers must be 0 .. 2^26-2");
    FmDev &d = h->d;
    h->iter = h->p.initialstep;
    h->simtime = h->p.simtime;
    fm::launch_reset_scalars(d, h->st);
    FM_CUDA(cudaMemsetAsync(d.cell_count, 0, sizeof(int32_t) * (size_t)d.ncell, h->st));
    d.n = n;
    if (n > 0) {
        const size_t n3 = 3 * (size_t)n;
        FM_CUDA(cudaMemcpyAsync(h->stage3, r, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
        FM_CUDA(cudaMemcpyAsync(h->stage3 + n3, v, sizeof(double) * n3, cudaMemcpyHostToDevice, h->st));
        fm::launch_scatter_state(d, h->stage3, h->stage3 + n3, nullptr, h->st);  // w = 0, a = 0
        FM_CUDA(cudaMemcpyAsync(d.slot_of, gid, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, h->st));
    }
    FM_CUDA(cudaGetLastError());
    FM_CUDA(cudaStreamSynchronize(h->st));
    h->n_own = n;
    h->n_halo = 0;
    h->dd_phase = 0;
    h->stage = 1;
    h->cells_valid = h->list_valid = false;
    h->has_pe = false;
    return FM_OK;
}

// Counts per destination rank from the device, their offsets back.
static int dd_fetch_counts(fm_handle *h, int32_t *counts, int *total)
{
    fm::DdDev &x = h->x;
    FM_CUDA(cudaMemcpyAsync(h->dd_counts.data(), x.count, sizeof(int32_t) * h->nranks, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    std::vector<int32_t> off((size_t)h->nranks);
    int t = 0;
    for (int r = 0; r < h->nranks; r++) {
        off[(size_t)r] = t;
        t += h->dd_counts[(size_t)r];
        if (counts) counts[r] = h->dd_counts[(size_t)r];
    }
    FM_CUDA(cudaMemcpyAsync(x.offset, off.data(), sizeof(int32_t) * h->nranks, cudaMemcpyHostToDevice, h->st));
    FM_CUDA(cudaMemsetAsync(x.cursor, 0, sizeof(int32_t) * h->nranks, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));  // `off` is a stack buffer
    *total = t;
    return FM_OK;
}

extern "C" int fm_dd_classify(fm_handle *h, int32_t wrap, int32_t *counts)
{
    FM_TRY(dd_ready(h, true, 1));
    if (!counts) return fail(FM_ERR_ARG, "null argument");
    FmDev &d = h->d;
    fm::DdDev &x = h->x;
    FM_CUDA(cudaMemsetAsync(d.cell_count, 0, sizeof(int32_t) * (size_t)d.ncell, h->st));
    FM_CUDA(cudaMemsetAsync(x.count, 0, sizeof(int32_t) * h->nranks, h->st));
    FM_CUDA(cudaMemsetAsync(x.nlist, 0, sizeof(int32_t), h->st));
    fm::launch_dd_classify(d, x, d.n, wrap ? 1 : 0, h->iter, h->st);
    h->launches += 1;
    FM_CUDA(cudaGetLastError());
    int total = 0;
    FM_TRY(dd_fetch_counts(h, counts, &total));
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    FM_TRY(status_error(h, s));
    h->n_kept = h->n_own - total;
    h->cells_valid = h->list_valid = false;
    h->dd_phase = 1;
    return FM_OK;
}

extern "C" int fm_dd_pack_emigrants(fm_handle *h, double *d_send)
{
    FM_TRY(dd_ready(h, true, 1));
    if (h->dd_phase != 1) return fail(FM_ERR_STATE, "fm_dd_pack_emigrants follows fm_dd_classify");
    int total = h->n_own - h->n_kept;
    if (total > 0 && !d_send) return fail(FM_ERR_ARG, "null send buffer");
    fm::launch_dd_pack_emigrants(h->d, h->x, total, d_send, h->st);
    h->launches += total > 0;
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

extern "C" int fm_dd_immigrate(fm_handle *h, const double *d_recv, int32_t n)
{
    FM_TRY(dd_ready(h, true, 1));
    if (h->dd_phase != 1) return fail(FM_ERR_STATE, "fm_dd_immigrate follows fm_dd_pack_emigrants");
    if (n < 0 || (n > 0 && !d_recv)) return fail(FM_ERR_ARG, "bad arrivals");
    FmDev &d = h->d;
    const int base = d.n;
    if ((int64_t)base + n > h->cap) return fail(FM_ERR_ARG, "arrivals exceed the subdomain's capacity");
    fm::launch_dd_append_immigrants(d, h->x, d_recv, n, base, h->iter, h->st);
    h->launches += n > 0;
    FM_CUDA(cudaGetLastError());
    h->n_pending = base + n;
    h->n_kept += n;
    h->dd_phase = 2;
    return FM_OK;
}

extern "C" int fm_dd_halo_counts(fm_handle *h, int32_t *counts)
{
    FM_TRY(dd_ready(h, true, 1));
    if (h->dd_phase != 2) return fail(FM_ERR_STATE, "fm_dd_halo_counts follows fm_dd_immigrate");
    if (!counts) return fail(FM_ERR_ARG, "null argument");
    FmDev d = h->d;
    FM_CUDA(cudaMemsetAsync(h->x.count, 0, sizeof(int32_t) * h->nranks, h->st));
    fm::launch_dd_halo_records(d, h->x, h->n_pending, 0, nullptr, h->st);
    h->launches += 1;
    FM_CUDA(cudaGetLastError());
    int total = 0;
    FM_TRY(dd_fetch_counts(h, counts, &total));
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    FM_TRY(status_error(h, s));
    h->dd_phase = 3;
    return FM_OK;
}

extern "C" int fm_dd_pack_halo(fm_handle *h, double *d_send)
{
    FM_TRY(dd_ready(h, true, 1));
    if (h->dd_phase != 3) return fail(FM_ERR_STATE, "fm_dd_pack_halo follows fm_dd_halo_counts");
    fm::launch_dd_halo_records(h->d, h->x, h->n_pending, 1, d_send, h->st);
    h->launches += 1;
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

// Neighbour rows of the sorted subdomain; a row overflow grows the rows and
// builds again.
static int dd_build(fm_handle *h)
{
    FmDev &d = h->d;
    for (int attempt = 0; attempt < 6; attempt++) {
        fm::launch_build_nlist(d, 0, h->iter, h->st);
        h->launches += 1;
        FM_CUDA(cudaGetLastError());
        fm::FmScalars s;
        FM_TRY(read_scalars(h, &s));
        if (!(s.status & fm::ST_NLIST) || (s.status & (fm::ST_FATAL & ~fm::ST_NLIST))) return status_error(h, s);
        const int want = round_up((int)std::ceil(1.2 * s.max_nbr) + 8, 8);
        if ((size_t)want * fm::nb_rows(h->cap) > ((size_t)1 << 34)) return status_error(h, s);
        FM_TRY(alloc_nlist(h, want));
        s.status &= ~fm::ST_NLIST;
        s.max_nbr = 0;
        FM_CUDA(cudaMemcpyAsync(&d.sc->status, &s.status, sizeof(uint32_t), cudaMemcpyHostToDevice, h->st));
        FM_CUDA(cudaMemcpyAsync(&d.sc->max_nbr, &s.max_nbr, sizeof(int32_t), cudaMemcpyHostToDevice, h->st));
        FM_CUDA(cudaStreamSynchronize(h->st));
    }
    return fail(FM_ERR_NLIST, "subdomain neighbour rows kept overflowing");
}

extern "C" int fm_dd_receive_halo(fm_handle *h, const double *d_recv, int32_t n)
{
    FM_TRY(dd_ready(h, true, 1));
    if (h->dd_phase != 3) return fail(FM_ERR_STATE, "fm_dd_receive_halo follows fm_dd_pack_halo");
    if (n < 0 || (n > 0 && !d_recv)) return fail(FM_ERR_ARG, "bad halo records");
    FmDev &d = h->d;
    const int base = h->n_pending;
    if ((int64_t)base + n > h->cap) return fail(FM_ERR_ARG, "halo copies exceed the subdomain's capacity");
    fm::launch_dd_append_halo(d, d_recv, n, base, h->st);
    // counting sort of every entry with a cell (owned kept, arrivals, halo
    // copies), in-cell by global number; then the rows
    FmDev old = d;
    old.n = base + n;
    fm::launch_scan_cells(old, 0, h->st);
    fm::launch_scatter(old, 0, h->st);
    d.n = h->n_kept + n;
    fm::launch_reorder(d, 0, h->tpos, h->tuidx, h->st);
    h->launches += 6;
    FM_CUDA(cudaGetLastError());
    h->n_own = h->n_kept;
    h->n_halo = n;
    h->cells_valid = true;
    d.nblocks_force = force_rows(h);
    FM_TRY(dd_build(h));
    h->list_valid = true;
    h->dd_phase = 0;
    if (h->stage < 2) h->stage = 2;
    return FM_OK;
}

extern "C" int fm_dd_counts(fm_handle *h, int32_t *n_owned, int32_t *n_halo)
{
    FM_TRY(dd_ready(h, false, 0));
    if (n_owned) *n_owned = h->n_own;
    if (n_halo) *n_halo = h->n_halo;
    return FM_OK;
}

extern "C" int fm_dd_cell_starts(fm_handle *h, int32_t *starts)
{
    FM_TRY(dd_ready(h, true, 2));
    if (!starts) return fail(FM_ERR_ARG, "null argument");
    FM_CUDA(cudaMemcpyAsync(starts, h->d.cell_start, sizeof(int32_t) * ((size_t)h->d.ncell + 1), cudaMemcpyDeviceToHost,
                            h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    return FM_OK;
}

extern "C" int fm_dd_gather_positions(fm_handle *h, const int32_t *d_idx, const int8_t *d_code, int32_t n,
                                      double *d_out)
{
    FM_TRY(dd_ready(h, true, 2));
    if (n < 0 || (n > 0 && (!d_idx || !d_code || !d_out))) return fail(FM_ERR_ARG, "bad gather list");
    fm::launch_dd_gather_positions(h->d, d_idx, d_code, n, d_out, h->st);
    h->launches += n > 0;
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

extern "C" int fm_dd_scatter_positions(fm_handle *h, const int32_t *d_idx, const double *d_in, int32_t n)
{
    FM_TRY(dd_ready(h, true, 2));
    if (n < 0 || (n > 0 && (!d_idx || !d_in))) return fail(FM_ERR_ARG, "bad scatter list");
    fm::launch_dd_scatter_positions(h->d, d_idx, d_in, n, h->st);
    h->launches += n > 0;
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

extern "C" int fm_dd_move1(fm_handle *h)
{
    FM_TRY(dd_ready(h, true, 2));
    fm::launch_move1(h->d, h->st);
    h->launches += 1;
    FM_CUDA(cudaGetLastError());
    return FM_OK;
}

extern "C" int fm_dd_vmax2(fm_handle *h, uint64_t *vmax2)
{
    FM_TRY(dd_ready(h, true, 2));
    if (!vmax2) return fail(FM_ERR_ARG, "null argument");
    unsigned long long v = 0ull;
    FM_CUDA(cudaMemcpyAsync(&v, &h->d.sc->vmax2, sizeof v, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    *vmax2 = (uint64_t)v;
    return FM_OK;
}

extern "C" int fm_dd_decide(fm_handle *h, uint64_t vmax2_global, int32_t iter, int32_t flip, int32_t *rebuild)
{
    FM_TRY(dd_ready(h, true, 2));
    if (!rebuild) return fail(FM_ERR_ARG, "null argument");
    const unsigned long long v = (unsigned long long)vmax2_global;
    FM_CUDA(cudaMemcpyAsync(&h->d.sc->vmax2, &v, sizeof v, cudaMemcpyHostToDevice, h->st));
    h->iter = iter;
    fm::launch_decide(h->d, iter, flip ? 1 : 0, h->p.rebuild_criteria, h->p.fixed_rebuild, h->half_min_delta, h->st);
    h->launches += 1;
    FM_CUDA(cudaGetLastError());
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));  // (also keeps `v` alive until the copy is done)
    FM_TRY(status_error(h, s));
    *rebuild = s.rebuild;
    return FM_OK;
}

extern "C" int fm_dd_forces(fm_handle *h, int32_t iter, int32_t record, int32_t mode)
{
    FM_TRY(dd_ready(h, true, 2));
    if (!(h->cells_valid && h->list_valid)) return fail(FM_ERR_STATE, "forces need a rebuild after the upload");
    if (mode < 0 || mode > 2) return fail(FM_ERR_ARG, "mode must be 0, 1 or 2");
    h->iter = iter;
    h->d.nblocks_force = force_rows(h);
    queue_force(h, record ? 1 : 0, mode);
    FM_CUDA(cudaGetLastError());
    if (record) h->has_pe = true;
    return FM_OK;
}

extern "C" int fm_dd_sums(fm_handle *h, double *sums)
{
    FM_TRY(dd_ready(h, true, 2));
    if (!sums) return fail(FM_ERR_ARG, "null argument");
    if (!h->has_pe) return fail(FM_ERR_STATE, "no record step has been computed");
    fm::launch_dd_sums(h->d, h->dd_sums, h->st);
    h->launches += 1;
    FM_CUDA(cudaGetLastError());
    FM_CUDA(cudaMemcpyAsync(sums, h->dd_sums, sizeof(double) * fm::RS_N, cudaMemcpyDeviceToHost, h->st));
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    FM_TRY(status_error(h, s));
    return FM_OK;
}

extern "C" int fm_dd_macro(fm_handle *h, const double *sums, int32_t iter, double simtime, fm_macro *out)
{
    FM_TRY(dd_ready(h, false, 0));
    if (!sums || !out) return fail(FM_ERR_ARG, "null argument");
    const FmDev &d = h->d;
    // evaluate_macroscopic_properties (simulation_record.f90:1205-1314), as the
    // single-system record kernel forms it, over the whole system's sums
    const double gnp = (double)h->p.np;
    fm_macro r;
    std::memset(&r, 0, sizeof r);
    r.iter = iter;
    r.simtime = simtime;
    r.vsum = sums[fm::RS_VSUM];
    r.mv2sum = sums[fm::RS_MV2];
    r.virial = sums[fm::RS_VIR];
    r.kinenergy = (0.5 * r.mv2sum) / gnp;
    r.potenergy = (0.5 * sums[fm::RS_PE]) / gnp + d.pot_slrc;
    r.totenergy = r.kinenergy + r.potenergy;
    r.temperature = r.mv2sum / (3.0 * gnp);
    r.pressure = (d.density / (gnp * 3.0)) * (r.mv2sum + r.virial / 2.0) + d.p_slrc;
    *out = r;
    if (sums[fm::RS_PEMAX] > 10000.0) return fail(FM_ERR_PE, "max(potenergymol) > 10000");
    return FM_OK;
}

extern "C" int fm_dd_download(fm_handle *h, int32_t cap, int32_t *n_owned, double *r, double *v, int32_t *gid)
{
    FM_TRY(dd_ready(h, false, 1));
    if (!n_owned) return fail(FM_ERR_ARG, "null argument");
    const FmDev &d = h->d;
    const size_t n = (size_t)d.n;
    std::vector<double4> pos(n);
    std::vector<double> vx(n), vy(n), vz(n);
    std::vector<int32_t> ids(n);
    fm::FmScalars s;
    FM_TRY(read_scalars(h, &s));
    if (n > 0) {
        FM_CUDA(cudaMemcpyAsync(pos.data(), fm::cur_pos(d, s.pset), sizeof(double4) * n, cudaMemcpyDeviceToHost, h->st));
        FM_CUDA(cudaMemcpyAsync(vx.data(), d.vx, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
        FM_CUDA(cudaMemcpyAsync(vy.data(), d.vy, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
        FM_CUDA(cudaMemcpyAsync(vz.data(), d.vz, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
        FM_CUDA(cudaMemcpyAsync(ids.data(), d.slot_of, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, h->st));
        FM_CUDA(cudaStreamSynchronize(h->st));
    }
    int m = 0;
    for (size_t i = 0; i < n; i++) {
        if (pos[i].w != 0.0) continue;  // halo copy
        if (m < cap) {
            if (r) { r[3 * m] = pos[i].x; r[3 * m + 1] = pos[i].y; r[3 * m + 2] = pos[i].z; }
            if (v) { v[3 * m] = vx[i]; v[3 * m + 1] = vy[i]; v[3 * m + 2] = vz[i]; }
            if (gid) gid[m] = ids[i];
        }
        m++;
    }
    *n_owned = m;
    if (m > cap) return fail(FM_ERR_ARG, "more owned molecules than cap");
    return FM_OK;
}

extern "C" int fm_dd_pair_list(fm_handle *h, int32_t *owner, int32_t *partner, int32_t *partner_cell, int64_t cap,
                               int64_t *n_out)
{
    FM_TRY(dd_ready(h, true, 2));
    if (!n_out) return fail(FM_ERR_ARG, "null output");
    const FmDev &d = h->d;
    const size_t n = (size_t)d.n;
    std::vector<int32_t> nnbr(n), slot(n), start((size_t)d.ncell + 1), nbr(fm::nb_rows((int)n) * (size_t)d.maxn);
    FM_CUDA(cudaMemcpyAsync(nnbr.data(), d.nnbr, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaMemcpyAsync(slot.data(), d.slot_of, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaMemcpyAsync(start.data(), d.cell_start, sizeof(int32_t) * start.size(), cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaMemcpyAsync(nbr.data(), d.nbr, sizeof(int32_t) * nbr.size(), cudaMemcpyDeviceToHost, h->st));
    FM_CUDA(cudaStreamSynchronize(h->st));
    int64_t k = 0;
    for (size_t i = 0; i < n; i++) {
        for (int q = 0; q < nnbr[i]; q++) {
            const int32_t j = nbr[fm::nb_row((int)i, d.maxn) + fm::nb_col(q)] & fm::NB_INDEX_MASK;
            if (k < cap) {
                if (owner) owner[k] = slot[i];
                if (partner) partner[k] = slot[(size_t)j];
                if (partner_cell)
                    partner_cell[k] = (int32_t)(std::upper_bound(start.begin(), start.end(), j) - start.begin()) - 1;
            }
            k++;
        }
    }
    *n_out = k;
    return FM_OK;
}
