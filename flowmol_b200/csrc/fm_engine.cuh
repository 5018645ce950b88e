// fm_engine.cuh -- device layout of the multi-job slot engine (batching and
// serving).  Many independent MD jobs share one arena of molecules, cells and
// neighbour-list rows; each job owns a slot with its own geometry, iteration
// counter, step budget, rebuild state and status.  A tick advances every
// resident job by one time step with a fixed sequence of kernels whose
// per-job decisions are taken on the device.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fm_common.cuh"

namespace fm {

enum : int { SLOT_EMPTY = 0, SLOT_SETUP = 1, SLOT_RUN = 2, SLOT_DONE = 3, SLOT_FAILED = 4 };
enum : int { PHASE_IDLE = 0, PHASE_SETUP = 1, PHASE_STEP = 2 };
enum : int { MODE_LIST = 1, MODE_ALLPAIRS = 2 };

// Molecular tags (modules.f90:79-88).
enum : int {
    TAG_FREE = 0, TAG_FIXED = 1, TAG_FIXED_SLIDE = 2, TAG_TETH = 3, TAG_THERMO = 4, TAG_TETH_THERMO = 5,
    TAG_TETH_SLIDE = 6, TAG_TETH_THERMO_SLIDE = 7
};

// Per-molecule record terms written on record ticks.
enum { RT_PE = 0, RT_VIR, RT_MV2, RT_VSUM, RT_PXX, RT_PYY, RT_PZZ, RT_PXY, RT_PXZ, RT_PYZ, RT_N };

struct EngSlot {
    // ---- static: written by the host at admission ----
    double L[3], hd[3], cs[3];
    int ne[3];
    int ncell, cell_off, cstart_off;  // cells [cell_off, +ncell); starts [cstart_off, +ncell+1)
    int mol_off, nmol;                // molecules [mol_off, +nmol)
    int64_t list_off;                 // neighbour rows start here, maxn entries per molecule
    int maxn;
    int build_blocks;                 // list build by 2x2x2 cells (sparse jobs), else by cell
    int tplot, integrator, ensemble, mode, pressure, nthermo, crit, fixed_rebuild;
    int iter0, nsteps;
    double rc2, rn2, potshift, half_min_delta, volume, density;
    double therm_T[2];
    double k2, k4, k6;
    // ---- dynamic: owned by the device while resident ----
    int state, phase, iter, pset;
    int rebuild, wrap, record, last;
    uint32_t status;
    int fail_iter;
    int rebuilds, nsamples;
    int max_nbr, pad_;
    unsigned long long vmax2;
    double rmax, simtime;
    double zeta[2], ascale[2], bscale[2];
    double ptensor[9];
    FmRecord last_rec;
};

// Per-tick summary written by the decide kernel, and the arena high-water
// marks written by the host at admission; kernels bound their loops and skip
// whole stages with them (device memory, so a captured graph sees updates).
struct EngFlags {
    int any_rebuild, any_list, any_ap, any_lfv, any_thermo, any_record;
    int mol_hwm, cell_hwm;
    // this tick's rebuilding jobs (slot order): count, their molecules, their
    // cells, their list-build units (cells or 2x2x2 blocks)
    int rb_n, rb_mtot, rb_ctot, rb_utot;
    // ticks run by the current launch of the tick loop (the graph's WHILE node),
    // and whether jobs wait in the host's queue (written before each launch)
    int loop_ticks, queue_waiting;
};

struct EngDev {
    int nslots;
    EngFlags *flags;
    int mol_cap;     // arena molecules
    int cell_cap;    // arena cells
    double dt, half_dt, half_dt2;
    int precision;
    EngSlot *slots;
    // molecules (arena order; a job's molecules are contiguous and re-ordered by cell inside it)
    double4 *pos0, *pos1;
    double *vx, *vy, *vz, *ax, *ay, *az;
    int32_t *slot_of;    // slot of a molecule, -1 = free
    int32_t *uidx;       // index of the molecule in its job's upload order
    int32_t *tag;
    double4 *rteth;      // tether anchor (x, y, z, unused)
    double4 *slidev;     // slide velocity (x, y, z, unused)
    // reorder scratch
    double4 *tpos, *trteth, *tslidev;
    double *tvx, *tvy, *tvz, *tax, *tay, *taz;
    int32_t *tuidx, *ttag;
    // cells
    int32_t *cell_slot;   // slot of an arena cell, -1 = free
    int32_t *cell_of;     // per molecule
    int32_t *cell_count;  // per cell
    int32_t *cell_start;  // per slot: ncell+1 absolute molecule indices
    int32_t *perm;        // new arena index -> old arena index
    // neighbour rows
    int32_t *nbr;
    int32_t *nnbr;
    // record terms and thermostat partials
    double *rterm;        // [mol][RT_N]
    double *tmv2;         // (v + a dt/2)^2 of thermostatted molecules, else 0
    // per-job reductions split over EY blocks: partial sums [slot][EY][RED_W]
    // and arrival counters [slot][2] (thermostat, record)
    double *red_part;
    int32_t *red_count;
    // rebuild work list of the tick: slots, and prefix sums of their molecules
    // and cells ([rb_n + 1] each), so the rebuild kernels visit only those
    int32_t *rb_slot, *rb_mpre, *rb_cpre, *rb_upre;
};

constexpr int EY = 16;      // blocks per job in the thermostat and record reductions
constexpr int RED_W = 24;   // doubles per partial: (sum, compensation) x up to 11 values, + max

__host__ __device__ inline double4 *eng_pos(const EngDev &d, int pset) { return pset ? d.pos1 : d.pos0; }

// Launch extents of a captured tick: the slot-indexed grids (one block row per
// slot) cover slots [0, slots), which must include every resident slot; the
// molecule and cell grids are grid-stride loops, so `mols` and `cells` only
// size them to the resident load (an empty block still costs launch time).
struct TickExtent {
    int slots, mols, cells;
};

// Launchers (fm_engine.cu); `tpm` = lanes per molecule of the force kernel.
void eng_tick(const EngDev &d, int tpm, const TickExtent &x, cudaStream_t st);
// The list build of the work list in d.flags / d.rb_* (autotuner timing runs).
void eng_build_only(const EngDev &d, int cells, cudaStream_t st);
void eng_force_only(const EngDev &d, int tpm, int mols, cudaStream_t st);  // autotuner: forces of running list jobs
void eng_scatter_job(const EngDev &d, int slot, int mol_off, int n, const double *r3, const double *v3,
                     const int32_t *tag, const double *rteth3, const double *slidev3, cudaStream_t st);
void eng_claim_cells(const EngDev &d, int slot, int cell_off, int ncell, cudaStream_t st);
void eng_gather_job(const EngDev &d, int slot, int mol_off, int n, double *r3, double *v3, cudaStream_t st);
void eng_release_job(const EngDev &d, int mol_off, int n, int cell_off, int ncell, cudaStream_t st);
int eng_kernels_per_tick();
// The tick loop's bookkeeping: the counter reset before the WHILE node, and
// the kernel that ends each iteration by setting the node's condition -- go
// on while some resident job runs and fewer than max_ticks ticks have run,
// unless a job has failed or has finished while others wait in the queue.
void eng_loop_reset(const EngDev &d, cudaStream_t st);
void eng_loop_continue(const EngDev &d, int slots, cudaGraphConditionalHandle cond, int body_ticks, int max_ticks,
                       cudaStream_t st);

}  // namespace fm
