// fm_engine_kernels.cu -- tick kernels of the multi-job slot engine.
//
// One tick advances every resident job by one step of its own integrator:
//   decide      per slot: set-up / advance / finish, rebuild check
//               (simulation_checkrebuild.f90:34,83-99), position-buffer flip
//   wrap+bin    sendmols wrap and assign_to_cell binning of rebuilding jobs
//   scan        per-slot exclusive scan of the cell counts
//   scatter     counting-sort placement, per-cell sort (deterministic order)
//   reorder     gather into cell order and copy back
//   build       neighbour rows (same pair set as the single-system build)
//   force       list jobs: LJ forces + the velocity-Verlet epilogue
//               (move(2), record terms, next move(1)) or, for leap-frog
//               jobs, a + record terms + thermostat partials
//   force_ap    all-pairs jobs (boxes below 3 cells): minimum image,
//               simulation_compute_forces_LJ_AP (simulation_compute_forces.f90:280-341)
//   thermo      per slot: Nose-Hoover wall thermostat update
//               (simulation_move_particles_lfv.f90:325-372)
//   move_lfv    leap-frog move with tags, tethers and sliding walls
//               (simulation_move_particles_lfv.f90:374-470, molecular_properties.f90:833-915)
//   record      per slot: macroscopic properties (simulation_record.f90:1205-1314) and the
//               virial pressure tensor (simulation_record.f90:3151-3220)
// Every kernel reads the slot table and does nothing for slots it does not
// concern, so the sequence is the same every tick and is captured once into a
// CUDA graph.  Jobs are independent: a job's arithmetic never depends on
// which other jobs are resident or where its molecules sit in the arena.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fm_device.cuh"
#include "fm_engine.cuh"
#include "fm_build.cuh"

namespace fm {

namespace {

constexpr int kSMs = 148;
inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }
inline int sgrid(long long n, int t, int per_sm) { return std::max(1, std::min(nblk(n, t), kSMs * per_sm)); }

__device__ __forceinline__ bool slot_active(const EngSlot &s)
{
    return s.phase != PHASE_IDLE && (s.status & ST_FATAL) == 0u;
}

__device__ __forceinline__ void slot_fail(EngSlot *s, uint32_t bit, int iter)
{
    uint32_t old = atomicOr(&s->status, bit);
    if ((old & ST_FATAL) == 0u) s->fail_iter = iter;
}

// Max of m2 over the lanes of a warp that belong to slot k, folded into the
// slot's vmax2 with one atomic when the whole warp is one job.
__device__ __forceinline__ void fold_vmax2(EngSlot *slots, int k, double m2)
{
    const int k0 = __shfl_sync(0xffffffffu, k, 0);
    if (__all_sync(0xffffffffu, k == k0 || k < 0)) {
        double w = warp_max(k >= 0 ? m2 : 0.0);
        if ((threadIdx.x & 31) == 0 && k0 >= 0 && w > 0.0)
            atomicMax(&slots[k0].vmax2, (unsigned long long)__double_as_longlong(w));
    } else if (k >= 0 && m2 > 0.0) {
        atomicMax(&slots[k].vmax2, (unsigned long long)__double_as_longlong(m2));
    }
}

// ---------------------------------------------------------------------------
// decide
// ---------------------------------------------------------------------------

__device__ void decide_slot(const EngDev &d, EngSlot &s)
{
    s.phase = PHASE_IDLE;
    if (s.state == SLOT_EMPTY || s.state == SLOT_DONE || s.state == SLOT_FAILED) return;
    if (s.status & ST_FATAL) { s.state = SLOT_FAILED; return; }
    if (s.state == SLOT_SETUP) {
        // setup: bin + list on the uploaded state (no wrap, md.f90:60-64); VV computes
        // the forces of iter0 (setup_initial_record.f90:88), leap-frog the first step
        s.state = SLOT_RUN;
        s.phase = PHASE_SETUP;
        s.rebuild = 1;
        s.wrap = 0;
        s.iter = s.integrator == 1 ? s.iter0 : s.iter0 + 1;
        s.record = (s.iter % s.tplot) == 0;
        s.last = s.iter == s.iter0 + s.nsteps;
        s.vmax2 = 0ull;
        s.rmax = 0.0;
        return;
    }
    // running: the previous tick computed the force of s.iter and wrote the next
    // positions (VV: move(1) of iter+1 unless it was the last; LF: the move of iter)
    const bool vv = s.integrator == 1;
    if (vv && s.iter == s.iter0 + s.nsteps) { s.state = SLOT_DONE; return; }
    s.pset ^= 1;
    int decide_iter = vv ? s.iter + 1 : s.iter;  // VV checks after move(1) of the new step
    if (!vv) s.simtime = s.simtime + d.dt;       // simulation_move_particles_lfv
    if (!vv && s.iter == s.iter0 + s.nsteps) { s.state = SLOT_DONE; return; }
    int rebuild = ((decide_iter + 1) % s.tplot) == 0 ? 1 : 0;
    if (s.crit == 0) {
        double vmax = sqrt(__longlong_as_double((long long)s.vmax2));
        s.rmax = __dadd_rn(s.rmax, __dmul_rn(vmax, d.dt));
        if (s.rmax > s.half_min_delta) rebuild = 1;
    } else if (s.crit == 1) {
        if ((decide_iter % s.fixed_rebuild) == 0) rebuild = 1;
    }
    s.vmax2 = 0ull;
    if (rebuild) { s.rmax = 0.0; s.rebuilds += 1; }
    s.iter = s.iter + 1;
    s.phase = PHASE_STEP;
    s.rebuild = rebuild;
    s.wrap = 1;
    s.record = (s.iter % s.tplot) == 0;
    s.last = s.iter == s.iter0 + s.nsteps;
    if (vv) s.simtime = s.simtime + d.dt;        // simulation_move_particles_vv.f90:191
}

__device__ __forceinline__ bool slot_rebuilding(const EngSlot &s) { return slot_active(s) && s.rebuild; }

constexpr int EDEC = 1024;
__global__ void __launch_bounds__(EDEC) k_e_decide(EngDev d)
{
    __shared__ int f[6];
    if (threadIdx.x < 6) f[threadIdx.x] = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < d.nslots; k += EDEC) {
        EngSlot &s = d.slots[k];
        decide_slot(d, s);
        if (slot_active(s)) {
            if (s.rebuild) atomicOr(&f[0], 1);
            if (s.mode == MODE_LIST) atomicOr(&f[1], 1);
            if (s.mode == MODE_ALLPAIRS) atomicOr(&f[2], 1);
            if (s.integrator == 0) atomicOr(&f[3], 1);
            if (s.integrator == 0 && s.nthermo > 0) atomicOr(&f[4], 1);
            if (s.record) atomicOr(&f[5], 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        d.flags->any_rebuild = f[0]; d.flags->any_list = f[1]; d.flags->any_ap = f[2];
        d.flags->any_lfv = f[3]; d.flags->any_thermo = f[4]; d.flags->any_record = f[5];
    }
    // rebuild work list in slot order: a block scan of (flag, molecules, cells)
    __shared__ int wsum[4][EDEC / 32];
    __shared__ int carry[4];
    if (threadIdx.x < 4) carry[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < d.nslots; base += EDEC) {
        const int k = base + threadIdx.x;
        int x[4] = {0, 0, 0, 0};
        if (k < d.nslots) {
            const EngSlot &s = d.slots[k];
            if (slot_rebuilding(s)) {
                x[0] = 1;
                x[1] = s.nmol;
                x[2] = s.mode == MODE_LIST ? s.ncell : 0;
                x[3] = s.mode != MODE_LIST ? 0
                       : s.build_blocks ? ((s.ne[0] + 1) / 2) * ((s.ne[1] + 1) / 2) * ((s.ne[2] + 1) / 2)
                                        : s.ncell;
            }
        }
        int incl[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            incl[q] = x[q];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl[q], o);
                if (lane >= o) incl[q] += t;
            }
            if (lane == 31) wsum[q][w] = incl[q];
        }
        __syncthreads();
        if (w == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int v = wsum[q][lane];
                int vi = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, vi, o);
                    if (lane >= o) vi += t;
                }
                wsum[q][lane] = vi - v;  // exclusive warp offsets
            }
        }
        __syncthreads();
        if (x[0]) {
            const int pos = carry[0] + wsum[0][w] + incl[0] - 1;
            d.rb_slot[pos] = k;
            d.rb_mpre[pos] = carry[1] + wsum[1][w] + incl[1] - x[1];
            d.rb_cpre[pos] = carry[2] + wsum[2][w] + incl[2] - x[2];
            d.rb_upre[pos] = carry[3] + wsum[3][w] + incl[3] - x[3];
        }
        __syncthreads();
        if (threadIdx.x == EDEC - 1)
            for (int q = 0; q < 4; q++) carry[q] += wsum[q][w] + incl[q];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        d.rb_mpre[carry[0]] = carry[1];
        d.rb_cpre[carry[0]] = carry[2];
        d.rb_upre[carry[0]] = carry[3];
        d.flags->rb_n = carry[0];
        d.flags->rb_mtot = carry[1];
        d.flags->rb_ctot = carry[2];
        d.flags->rb_utot = carry[3];
    }
}

// Grid-stride over the tick's rebuild work list: element g of [0, total) is
// entry r (advanced as g grows) at offset g - pre[r].
__device__ __forceinline__ int rb_entry(const int32_t *pre, int g, int &r)
{
    while (g >= pre[r + 1]) r++;
    return g - pre[r];
}

// ---------------------------------------------------------------------------
// rebuild pipeline (gated per slot)
// ---------------------------------------------------------------------------


__global__ void k_e_wrap_bin(EngDev d)
{
    if (!d.flags->any_rebuild) return;
    const int tot = d.flags->rb_mtot;
    int r = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < tot; g += gridDim.x * blockDim.x) {
        const int off = rb_entry(d.rb_mpre, g, r);
        EngSlot &s = d.slots[d.rb_slot[r]];
        const int i = s.mol_off + off;
        double4 *P = eng_pos(d, s.pset);
        double4 p = P[i];
        if (s.wrap) {
            double4 q = p;
            if (q.x >= s.hd[0]) q.x = __dsub_rn(q.x, s.L[0]);
            if (q.x < -s.hd[0]) q.x = __dadd_rn(q.x, s.L[0]);
            if (q.y >= s.hd[1]) q.y = __dsub_rn(q.y, s.L[1]);
            if (q.y < -s.hd[1]) q.y = __dadd_rn(q.y, s.L[1]);
            if (q.z >= s.hd[2]) q.z = __dsub_rn(q.z, s.L[2]);
            if (q.z < -s.hd[2]) q.z = __dadd_rn(q.z, s.L[2]);
            if (q.x != p.x || q.y != p.y || q.z != p.z) {
                P[i] = q;
                // tether anchors follow their molecule across the boundary (messenger.serial.f90:975)
                double4 t = d.rteth[i];
                if (q.x != p.x) t.x = q.x < p.x ? __dsub_rn(t.x, s.L[0]) : __dadd_rn(t.x, s.L[0]);
                if (q.y != p.y) t.y = q.y < p.y ? __dsub_rn(t.y, s.L[1]) : __dadd_rn(t.y, s.L[1]);
                if (q.z != p.z) t.z = q.z < p.z ? __dsub_rn(t.z, s.L[2]) : __dadd_rn(t.z, s.L[2]);
                d.rteth[i] = t;
            }
            p = q;
        }
        if (s.mode != MODE_LIST) continue;
        bool bad = false;
        int cx = bin_axis(p.x, s.hd[0], s.cs[0], s.ne[0], bad);
        int cy = bin_axis(p.y, s.hd[1], s.cs[1], s.ne[1], bad);
        int cz = bin_axis(p.z, s.hd[2], s.cs[2], s.ne[2], bad);
        if (bad) slot_fail(&s, ST_ESCAPE, s.iter);
        int c = s.cell_off + cx + s.ne[0] * (cy + s.ne[1] * cz);
        d.cell_of[i] = c;
        atomicAdd(&d.cell_count[c], 1);
    }
}

constexpr int ESCAN = 1024;
__global__ void __launch_bounds__(ESCAN) k_e_scan(EngDev d)
{
    if (!d.flags->any_rebuild) return;
    const EngSlot &s = d.slots[blockIdx.x];
    if (!slot_rebuilding(s) || s.mode != MODE_LIST) return;
    __shared__ int ws[ESCAN / 32];
    __shared__ int carry_s;
    if (threadIdx.x == 0) carry_s = s.mol_off;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < s.ncell; base += ESCAN) {
        const int c = base + threadIdx.x;
        const int v = c < s.ncell ? d.cell_count[s.cell_off + c] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) ws[w] = incl;
        __syncthreads();
        if (w == 0) {
            int x = ws[lane], xi = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, xi, o);
                if (lane >= o) xi += t;
            }
            ws[lane] = xi - x;
        }
        __syncthreads();
        const int carry = carry_s;
        if (c < s.ncell) {
            d.cell_start[s.cstart_off + c] = carry + ws[w] + incl - v;
            d.cell_count[s.cell_off + c] = 0;
        }
        __syncthreads();
        if (threadIdx.x == ESCAN - 1) carry_s = carry + ws[w] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) d.cell_start[s.cstart_off + s.ncell] = carry_s;
}

__global__ void k_e_scatter(EngDev d)
{
    if (!d.flags->any_rebuild) return;
    const int tot = d.flags->rb_mtot;
    int r = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < tot; g += gridDim.x * blockDim.x) {
        const int off = rb_entry(d.rb_mpre, g, r);
        const EngSlot &s = d.slots[d.rb_slot[r]];
        if (s.mode != MODE_LIST) continue;
        const int i = s.mol_off + off;
        const int c = d.cell_of[i];
        const int slot = d.cell_start[s.cstart_off + (c - s.cell_off)] + atomicAdd(&d.cell_count[c], 1);
        d.perm[slot] = i;
    }
}

__global__ void k_e_sort(EngDev d)
{
    if (!d.flags->any_rebuild) return;
    const int tot = d.flags->rb_ctot;
    int r = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < tot; g += gridDim.x * blockDim.x) {
        const int lc = rb_entry(d.rb_cpre, g, r);
        const EngSlot &s = d.slots[d.rb_slot[r]];
        const int c = s.cell_off + lc;
        const int b = d.cell_start[s.cstart_off + lc], e = d.cell_start[s.cstart_off + lc + 1];
        for (int x = b + 1; x < e; x++) {
            int key = d.perm[x];
            int y = x - 1;
            while (y >= b && d.perm[y] > key) {
                d.perm[y + 1] = d.perm[y];
                y--;
            }
            d.perm[y + 1] = key;
        }
        d.cell_count[c] = 0;
    }
}

__global__ void k_e_reorder_gather(EngDev d)
{
    if (!d.flags->any_rebuild) return;
    const int tot = d.flags->rb_mtot;
    int r = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < tot; g += gridDim.x * blockDim.x) {
        const int off = rb_entry(d.rb_mpre, g, r);
        const EngSlot &s = d.slots[d.rb_slot[r]];
        if (s.mode != MODE_LIST) continue;
        const int n = s.mol_off + off;
        const int o = d.perm[n];
        d.tpos[n] = eng_pos(d, s.pset)[o];
        d.tvx[n] = d.vx[o]; d.tvy[n] = d.vy[o]; d.tvz[n] = d.vz[o];
        d.tax[n] = d.ax[o]; d.tay[n] = d.ay[o]; d.taz[n] = d.az[o];
        d.tuidx[n] = d.uidx[o];
        d.ttag[n] = d.tag[o];
        d.trteth[n] = d.rteth[o];
        d.tslidev[n] = d.slidev[o];
    }
}

__global__ void k_e_reorder_copy(EngDev d)
{
    if (!d.flags->any_rebuild) return;
    const int tot = d.flags->rb_mtot;
    int r = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < tot; g += gridDim.x * blockDim.x) {
        const int off = rb_entry(d.rb_mpre, g, r);
        const EngSlot &s = d.slots[d.rb_slot[r]];
        if (s.mode != MODE_LIST) continue;
        const int n = s.mol_off + off;
        eng_pos(d, s.pset)[n] = d.tpos[n];
        d.vx[n] = d.tvx[n]; d.vy[n] = d.tvy[n]; d.vz[n] = d.tvz[n];
        d.ax[n] = d.tax[n]; d.ay[n] = d.tay[n]; d.az[n] = d.taz[n];
        d.uidx[n] = d.tuidx[n];
        d.tag[n] = d.ttag[n];
        d.rteth[n] = d.trteth[n];
        d.slidev[n] = d.tslidev[n];
    }
}

// Neighbour rows of the tick's rebuilding jobs, one warp per work unit (a
// cell, or a block of 2x2x2 cells for sparse jobs): the single-system
// routines (build_cell / build_block, fm_build.cuh: pair set of
// assign_to_neighbourlist_halfint_opt, linklist.f90:660-804) on the unit's job.
__global__ void __launch_bounds__(NB_THREADS, 6) k_e_build(EngDev d)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    union WarpShared {
        BuildShared<false> cell;
        BlockShared<false> block;
    };
    __shared__ WarpShared sh[NB_WARPS];
    __shared__ CellSys ys[NB_WARPS];  // the unit's job, read through shared memory
    if (!d.flags->any_rebuild) return;
    const int tot = d.flags->rb_utot;
    int r = 0, r_loaded = -1;
    for (int g = blockIdx.x * NB_WARPS + warp; g < tot; g += gridDim.x * NB_WARPS) {
        const int unit = rb_entry(d.rb_upre, g, r);
        EngSlot &s = d.slots[d.rb_slot[r]];
        __syncwarp();
        if (r != r_loaded && lane == 0) {
            CellSys &y = ys[warp];
            y.P = eng_pos(d, s.pset) + s.mol_off;
            y.cell_start = d.cell_start + s.cstart_off;
            y.mol_off = s.mol_off;
            for (int q = 0; q < 3; q++) { y.ne[q] = s.ne[q]; y.cs[q] = s.cs[q]; y.hd[q] = s.hd[q]; y.L[q] = s.L[q]; }
            y.rn2 = s.rn2;
            y.nbr = d.nbr + s.list_off;
            y.nnbr = d.nnbr + s.mol_off;
            y.maxn = s.maxn;
            y.max_nbr = &s.max_nbr;
            y.chain = y.subchain = nullptr;
            y.bflag = nullptr;
            y.bnd = y.nbond = nullptr;
            y.dd = 0;
            y.org[0] = y.org[1] = y.org[2] = 0;
        }
        __syncwarp();
        r_loaded = r;
        // a cell or, for sparse jobs, a block of 2x2x2 cells: the same rows
        const uint32_t over = s.build_blocks ? build_block<false>(ys[warp], unit, sh[warp].block, lane)
                                             : build_cell<false>(ys[warp], unit, sh[warp].cell, lane);
        if (lane == 0 && (over & BUILD_OVER_LIST)) slot_fail(&s, ST_NLIST, s.iter);
    }
}

// ---------------------------------------------------------------------------
// forces and the integrator epilogue
// ---------------------------------------------------------------------------

struct PairAcc {
    double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0, vir = 0.0;
    double rxx = 0.0, ryy = 0.0, rzz = 0.0, rxy = 0.0, rxz = 0.0, ryz = 0.0;  // sum acc * rij (x) rij
};

template <int PREC>
__device__ __forceinline__ void lj_pair(PairAcc &a, double dx, double dy, double dz, double r2, double potshift,
                                        bool rec, bool ptens)
{
    if (PREC == 0) {
        const double s = __drcp_rn(r2), s2 = s * s, s4 = s2 * s2;  // == 1.0 / r2
        const double acc = 48.0 * (s4 * s2 * s - 0.5 * s4);
        a.fx += acc * dx; a.fy += acc * dy; a.fz += acc * dz;
        if (rec) {
            const double s3 = s2 * s;
            a.pe += 4.0 * (s3 * s3 - s3) - potshift;
            a.vir += acc * r2;
            if (ptens) {  // pressure_tensor_forces (simulation_record.f90:6239-6256)
                a.rxx += acc * dx * dx; a.ryy += acc * dy * dy; a.rzz += acc * dz * dz;
                a.rxy += acc * dx * dy; a.rxz += acc * dx * dz; a.ryz += acc * dy * dz;
            }
        }
    } else {
        // FP32 pair magnitude; the FP64 rij scales it (one conversion)
        const float s = rcp_f32((float)r2), s2 = s * s, s4 = s2 * s2;
        const double acc = (double)(48.0f * (s4 * s2 * s - 0.5f * s4));
        a.fx = fma(acc, dx, a.fx); a.fy = fma(acc, dy, a.fy); a.fz = fma(acc, dz, a.fz);
        if (rec) {
            const float s3 = s2 * s;
            a.pe += (double)(4.0f * (s3 * s3 - s3)) - potshift;
            a.vir += acc * r2;
            if (ptens) {
                a.rxx += acc * dx * dx; a.ryy += acc * dy * dy; a.rzz += acc * dz * dz;
                a.rxy += acc * dx * dy; a.rxz += acc * dx * dz; a.ryz += acc * dy * dz;
            }
        }
    }
}

__device__ __forceinline__ void reduce_lanes(PairAcc &a, int tpm, bool rec, bool ptens)
{
    for (int o = tpm / 2; o > 0; o >>= 1) {
        a.fx += __shfl_xor_sync(0xffffffffu, a.fx, o);
        a.fy += __shfl_xor_sync(0xffffffffu, a.fy, o);
        a.fz += __shfl_xor_sync(0xffffffffu, a.fz, o);
        if (rec) {
            a.pe += __shfl_xor_sync(0xffffffffu, a.pe, o);
            a.vir += __shfl_xor_sync(0xffffffffu, a.vir, o);
            if (ptens) {
                a.rxx += __shfl_xor_sync(0xffffffffu, a.rxx, o);
                a.ryy += __shfl_xor_sync(0xffffffffu, a.ryy, o);
                a.rzz += __shfl_xor_sync(0xffffffffu, a.rzz, o);
                a.rxy += __shfl_xor_sync(0xffffffffu, a.rxy, o);
                a.rxz += __shfl_xor_sync(0xffffffffu, a.rxz, o);
                a.ryz += __shfl_xor_sync(0xffffffffu, a.ryz, o);
            }
        }
    }
}

__device__ __forceinline__ bool thermo_tag(int t)
{
    return t == TAG_THERMO || t == TAG_TETH_THERMO || t == TAG_TETH_THERMO_SLIDE;
}

// Epilogue for molecule i of slot s with its summed pair forces; returns |v|^2
// after a velocity-Verlet move(1) (0 otherwise).
__device__ __forceinline__ double epilogue(const EngDev &d, const EngSlot &s, int i, const PairAcc &a)
{
    const double fx = a.fx, fy = a.fy, fz = a.fz;
    d.ax[i] = fx; d.ay[i] = fy; d.az[i] = fz;
    double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
    double m2 = 0.0;
    double wx, wy, wz;  // velocity the record uses
    if (s.integrator == 1) {
        if (s.phase == PHASE_STEP) {  // move(2)
            vx = __dadd_rn(vx, __dmul_rn(d.half_dt, fx));
            vy = __dadd_rn(vy, __dmul_rn(d.half_dt, fy));
            vz = __dadd_rn(vz, __dmul_rn(d.half_dt, fz));
        }
        wx = vx; wy = vy; wz = vz;
    } else {
        // leap-frog records v + a dt/2 (simulation_record.f90:1243)
        wx = __dadd_rn(vx, __dmul_rn(__dmul_rn(0.5, fx), d.dt));
        wy = __dadd_rn(vy, __dmul_rn(__dmul_rn(0.5, fy), d.dt));
        wz = __dadd_rn(vz, __dmul_rn(__dmul_rn(0.5, fz), d.dt));
        if (s.nthermo > 0) d.tmv2[i] = thermo_tag(d.tag[i]) ? norm2_rn(wx, wy, wz) : 0.0;
    }
    if (s.record) {
        double *t = d.rterm + (size_t)i * RT_N;
        t[RT_PE] = a.pe;
        t[RT_VIR] = a.vir;
        t[RT_MV2] = norm2_rn(wx, wy, wz);
        t[RT_VSUM] = __dadd_rn(__dadd_rn(wx, wy), wz);
        if (s.pressure) {  // Pxymol = v (x) v + rfmol/2 (simulation_record.f90:3170-3201)
            t[RT_PXX] = wx * wx + 0.5 * a.rxx; t[RT_PYY] = wy * wy + 0.5 * a.ryy;
            t[RT_PZZ] = wz * wz + 0.5 * a.rzz; t[RT_PXY] = wx * wy + 0.5 * a.rxy;
            t[RT_PXZ] = wx * wz + 0.5 * a.rxz; t[RT_PYZ] = wy * wz + 0.5 * a.ryz;
        }
    }
    if (s.integrator == 1) {
        if (!s.last) {  // move(1) of the next step into the other position buffer
            double4 p = eng_pos(d, s.pset)[i];
            p.x = __dadd_rn(__dadd_rn(p.x, __dmul_rn(d.dt, vx)), __dmul_rn(d.half_dt2, fx));
            p.y = __dadd_rn(__dadd_rn(p.y, __dmul_rn(d.dt, vy)), __dmul_rn(d.half_dt2, fy));
            p.z = __dadd_rn(__dadd_rn(p.z, __dmul_rn(d.dt, vz)), __dmul_rn(d.half_dt2, fz));
            vx = __dadd_rn(vx, __dmul_rn(d.half_dt, fx));
            vy = __dadd_rn(vy, __dmul_rn(d.half_dt, fy));
            vz = __dadd_rn(vz, __dmul_rn(d.half_dt, fz));
            eng_pos(d, s.pset ^ 1)[i] = p;
            m2 = norm2_rn(vx, vy, vz);
        }
        d.vx[i] = vx; d.vy[i] = vy; d.vz[i] = vz;
    }
    return m2;
}

constexpr int EF_THREADS = 256;

// Two launches per tick: REC false takes the molecules of jobs that do not
// record this tick (forces only: few registers, full occupancy), REC true the
// recording ones (PE, virial and the pressure-tensor terms as well).
template <int TPM, int PREC, bool FORCE_ONLY, bool REC>
__global__ void __launch_bounds__(EF_THREADS, REC ? 2 : 4) k_e_force(EngDev d)
{
    constexpr int PER_BLOCK = EF_THREADS / TPM;
    const int lane = threadIdx.x % TPM;
    if (!FORCE_ONLY && !d.flags->any_list) return;
    if (REC && !d.flags->any_record) return;
    const int hwm = d.flags->mol_hwm;
    for (int base = blockIdx.x * PER_BLOCK; base < hwm; base += gridDim.x * PER_BLOCK) {
        const int i = base + threadIdx.x / TPM;
        int k = i < hwm ? d.slot_of[i] : -1;
        const EngSlot *sp = k >= 0 ? &d.slots[k] : nullptr;
        bool act = k >= 0 && sp->mode == MODE_LIST &&
                   (FORCE_ONLY ? (sp->state == SLOT_RUN) : slot_active(*sp));
        if (!FORCE_ONLY && act && (sp->record != 0) != REC) act = false;
        if (!act) k = -1;
        const bool rec = REC && act;
        const bool ptens = rec && sp->pressure;
        PairAcc a;
        if (act) {
            const EngSlot &s = *sp;
            const double4 *P = eng_pos(d, s.pset);
            const double4 pi = P[i];
            const int cnt = d.nnbr[i];
            const int32_t *L = d.nbr + s.list_off + nb_row(i - s.mol_off, s.maxn);
            const double4 *Pj = P + s.mol_off;
            for (int k0 = lane * 4; k0 < cnt; k0 += 4 * TPM) {
                const int4 e4 = ld_stream_int4(reinterpret_cast<const int4 *>(L + nb_col(k0)));
                const int ev[4] = {e4.x, e4.y, e4.z, e4.w};
                double4 pj[4];
#pragma unroll
                for (int q = 0; q < 4; q++)
                    if (k0 + q < cnt) pj[q] = ldg_pos(Pj + (ev[q] & NB_INDEX_MASK));
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (k0 + q >= cnt) break;
                    const int code = ev[q] >> NB_SHIFT_BITS;
                    double xj = pj[q].x, yj = pj[q].y, zj = pj[q].z;
                    if (code != NB_NOSHIFT) {  // rows of boundary cells only
                        xj = image(xj, (code & 3) - 1, s.L[0]);
                        yj = image(yj, ((code >> 2) & 3) - 1, s.L[1]);
                        zj = image(zj, ((code >> 4) & 3) - 1, s.L[2]);
                    }
                    const double dx = __dsub_rn(pi.x, xj);
                    const double dy = __dsub_rn(pi.y, yj);
                    const double dz = __dsub_rn(pi.z, zj);
                    const double r2 = norm2_rn(dx, dy, dz);
                    if (r2 < s.rc2) lj_pair<PREC>(a, dx, dy, dz, r2, s.potshift, rec, ptens);
                }
            }
        }
        // lanes of one molecule share the reduction; record flags are per molecule but
        // the lanes of a group agree, and inactive lanes add zeros
        const bool any_rec = __any_sync(0xffffffffu, rec);
        const bool any_pt = __any_sync(0xffffffffu, ptens);
        reduce_lanes(a, TPM, any_rec, any_pt);
        double m2 = 0.0;
        if (act && lane == 0) {
            if (FORCE_ONLY) { d.ax[i] = a.fx; d.ay[i] = a.fy; d.az[i] = a.fz; }
            else m2 = epilogue(d, *sp, i, a);
        }
        if (!FORCE_ONLY) fold_vmax2(d.slots, lane == 0 ? k : -1, m2);
    }
}

// All pairs with per-axis minimum image for jobs below 3 cells per axis
// (simulation_compute_forces_LJ_AP, simulation_compute_forces.f90:280-341).
// Blocks (EAP_XBLOCKS x EAP_YBLOCKS; x strides over the slots), one warp per
// molecule of an all-pairs job: lane l takes partners mol_off + l, + 32, ...
// and the lanes' sums are combined in a fixed order.
constexpr int EAP_THREADS = 256;
constexpr int EAP_XBLOCKS = 32, EAP_YBLOCKS = 16;
template <int PREC>
__global__ void __launch_bounds__(EAP_THREADS) k_e_force_ap(EngDev d)
{
    if (!d.flags->any_ap) return;
    for (int k = blockIdx.x; k < d.nslots; k += gridDim.x) {
    const EngSlot &s = d.slots[k];
    if (s.mode != MODE_ALLPAIRS || !slot_active(s)) continue;  // uniform per block
    const int lane = threadIdx.x & 31;
    const double4 *P = eng_pos(d, s.pset);
    // simulation_compute_forces_LJ_AP (:280-341) calls no pressure_tensor_forces:
    // an all-pairs job's pressure tensor has the kinetic part only
    const bool rec = s.record, ptens = false;
    constexpr int WPB = EAP_THREADS / 32;
    for (int i = s.mol_off + blockIdx.y * WPB + (threadIdx.x >> 5); i < s.mol_off + s.nmol;
         i += EAP_YBLOCKS * WPB) {
        const double4 pi = P[i];
        PairAcc a;
        for (int j = s.mol_off + lane; j < s.mol_off + s.nmol; j += 32) {
            if (j == i) continue;
            const double4 pj = ldg_pos(P + j);
            double r[3] = {__dsub_rn(pi.x, pj.x), __dsub_rn(pi.y, pj.y), __dsub_rn(pi.z, pj.z)};
            double r2 = 0.0;
#pragma unroll
            for (int q = 0; q < 3; q++) {
                if (fabs(r[q]) > s.hd[q]) r[q] = __dsub_rn(r[q], copysign(s.L[q], r[q]));
                r2 = __dadd_rn(r2, __dmul_rn(r[q], r[q]));
            }
            if (r2 < s.rc2) lj_pair<PREC>(a, r[0], r[1], r[2], r2, s.potshift, rec, ptens);
        }
        reduce_lanes(a, 32, rec, ptens);
        double m2 = 0.0;
        if (lane == 0) m2 = epilogue(d, s, i, a);
        fold_vmax2(d.slots, lane == 0 ? k : -1, m2);
    }
    }
}

// ---------------------------------------------------------------------------
// thermostat, leap-frog move, records
// ---------------------------------------------------------------------------

constexpr int ER = 256;

// (s, c) += (s2, c2): Neumaier merge of two compensated partial sums.
__device__ __forceinline__ void nmerge(double &s, double &c, double s2, double c2)
{
    neumaier(s, c, s2);
    c += c2;
}

// Compensated sums of NV values over the block, in a fixed tree order (warp
// xor tree, then the warps in index order); the result is in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (&c)[NV])
{
    __shared__ double sv[NV][ER / 32], sc[NV][ER / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NV; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double s2 = __shfl_xor_sync(0xffffffffu, v[k], o), c2 = __shfl_xor_sync(0xffffffffu, c[k], o);
            nmerge(v[k], c[k], s2, c2);
        }
        if (l == 0) { sv[k][w] = v[k]; sc[k][w] = c[k]; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < NV; k++) {
            double s = sv[k][0], cc = sc[k][0];
            for (int q = 1; q < ER / 32; q++) nmerge(s, cc, sv[k][q], sc[k][q]);
            v[k] = s; c[k] = cc;
        }
    }
    __syncthreads();
}

// Block y of EY over a job's molecules: [lo, hi) of [mol_off, mol_off + nmol).
__device__ __forceinline__ void job_chunk(const EngSlot &s, int y, int &lo, int &hi)
{
    const int chunk = (s.nmol + EY - 1) / EY;
    lo = s.mol_off + min(s.nmol, y * chunk);
    hi = s.mol_off + min(s.nmol, (y + 1) * chunk);
}

// Publishes block y's NV compensated sums (and a max) for slot k; the last of
// the EY blocks to arrive merges all partials in y order into (v, c, mx) and
// returns true (in thread 0 only).  The merge order does not depend on which
// block arrives last, so the result is deterministic.
template <int NV>
__device__ bool job_merge(const EngDev &d, int k, int which, double (&v)[NV], double (&c)[NV], double &mx)
{
    __shared__ bool last;
    double *part = d.red_part + ((size_t)k * EY + blockIdx.y) * RED_W;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NV; q++) { part[2 * q] = v[q]; part[2 * q + 1] = c[q]; }
        part[2 * NV] = mx;
        __threadfence();
        const int prev = atomicAdd(&d.red_count[2 * k + which], 1);
        last = prev == EY - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return false;
    __threadfence();
    const volatile double *all = d.red_part + (size_t)k * EY * RED_W;
    for (int q = 0; q < NV; q++) { v[q] = all[2 * q]; c[q] = all[2 * q + 1]; }
    mx = all[2 * NV];
    for (int y = 1; y < EY; y++) {
        const volatile double *py = all + (size_t)y * RED_W;
        for (int q = 0; q < NV; q++) nmerge(v[q], c[q], py[2 * q], py[2 * q + 1]);
        mx = fmax(mx, py[2 * NV]);
    }
    d.red_count[2 * k + which] = 0;  // ready for the next tick
    return true;
}

// Nose-Hoover on thermostatted molecules per region (nthermo = 1, or 2 split
// at y = 0): Q = N_thermo dt, dzeta/dt = (sum m v^2 - (3 N_thermo + 1) T)/Q.
// Grid (slot, EY).
__global__ void __launch_bounds__(ER) k_e_thermo(EngDev d)
{
    if (!d.flags->any_thermo) return;
    const int k = blockIdx.x;
    EngSlot &s = d.slots[k];
    if (!slot_active(s) || s.integrator != 0 || s.nthermo <= 0) return;
    double v[4] = {0, 0, 0, 0}, c[4] = {0, 0, 0, 0};  // mv2 region 0/1, count region 0/1
    const double4 *P = eng_pos(d, s.pset);
    int lo, hi;
    job_chunk(s, blockIdx.y, lo, hi);
    for (int i = lo + threadIdx.x; i < hi; i += ER) {
        if (!thermo_tag(d.tag[i])) continue;
        const int tr = (s.nthermo == 2 && !(P[i].y > 0.0)) ? 1 : 0;
        neumaier(v[tr], c[tr], d.tmv2[i]);
        neumaier(v[2 + tr], c[2 + tr], 1.0);
    }
    block_sum<4>(v, c);
    double mx = 0.0;
    if (!job_merge<4>(d, k, 0, v, c, mx)) return;
    for (int r = 0; r < s.nthermo; r++) {
        const double np_t = v[2 + r] + c[2 + r];
        const double Q = 1.0 * np_t * d.dt;
        const double dzeta = np_t > 0.0 ? ((v[r] + c[r]) - (3.0 * np_t + 1.0) * s.therm_T[r]) / Q : 0.0;
        s.zeta[r] = s.zeta[r] + d.dt * dzeta;
        s.bscale[r] = 1.0 / (1.0 + 0.5 * d.dt * s.zeta[r]);
        s.ascale[r] = (1.0 - 0.5 * d.dt * s.zeta[r]) * s.bscale[r];
    }
}

__global__ void k_e_move_lfv(EngDev d)
{
    if (!d.flags->any_lfv) return;
    const int hwm = d.flags->mol_hwm;
    for (int base = blockIdx.x * blockDim.x; base < hwm; base += gridDim.x * blockDim.x) {
        const int i = base + threadIdx.x;
        int k = i < hwm ? d.slot_of[i] : -1;
        const EngSlot *sp = k >= 0 ? &d.slots[k] : nullptr;
        const bool act = k >= 0 && sp->integrator == 0 && slot_active(*sp);
        if (!act) k = -1;
        double m2 = 0.0;
        if (act) {
            const EngSlot &s = *sp;
            const double dt = d.dt;
            double4 p = eng_pos(d, s.pset)[i];
            double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
            double ax = d.ax[i], ay = d.ay[i], az = d.az[i];
            const int tag = s.ensemble == 6 ? d.tag[i] : TAG_FREE;
            const bool teth = tag == TAG_TETH || tag == TAG_TETH_THERMO || tag == TAG_TETH_SLIDE ||
                              tag == TAG_TETH_THERMO_SLIDE;
            const bool slide = tag == TAG_FIXED_SLIDE || tag == TAG_TETH_SLIDE || tag == TAG_TETH_THERMO_SLIDE;
            const double4 sv = slide || teth ? d.slidev[i] : make_double4(0, 0, 0, 0);
            if (teth) {  // tether_force (molecular_properties.f90:833-915), polynomial form
                double4 rt = d.rteth[i];
                const double rx = p.x - rt.x, ry = p.y - rt.y, rz = p.z - rt.z;
                const double mag = sqrt(rx * rx + ry * ry + rz * rz);
                const double mag2 = mag * mag;
                const double acct = -2.0 * s.k2 * mag - 4.0 * s.k4 * mag2 - 6.0 * s.k6 * (mag2 * mag2);
                ax = ax + acct * rx; ay = ay + acct * ry; az = az + acct * rz;
                rt.x = rt.x + sv.x * dt; rt.y = rt.y + sv.y * dt; rt.z = rt.z + sv.z * dt;
                d.rteth[i] = rt;
                d.ax[i] = ax; d.ay[i] = ay; d.az[i] = az;
            }
            if (tag == TAG_FIXED) {
                // fixed: neither r nor v changes
            } else if (tag == TAG_FIXED_SLIDE) {
                p.x = p.x + dt * sv.x; p.y = p.y + dt * sv.y; p.z = p.z + dt * sv.z;
            } else if (thermo_tag(tag)) {
                const int tr = (s.nthermo == 2 && !(p.y > 0.0)) ? 1 : 0;
                const double as = s.ascale[tr], bs = s.bscale[tr];
                vx = vx * as + ax * dt * bs; p.x = p.x + vx * dt;
                vy = vy * as + ay * dt * bs; p.y = p.y + vy * dt;
                vz = vz * as + az * dt * bs; p.z = p.z + vz * dt;
                if (tag == TAG_TETH_THERMO_SLIDE) { p.x = p.x + sv.x * dt; p.y = p.y + sv.y * dt; p.z = p.z + sv.z * dt; }
            } else {
                vx = vx + dt * ax; vy = vy + dt * ay; vz = vz + dt * az;
                p.x = p.x + dt * vx; p.y = p.y + dt * vy; p.z = p.z + dt * vz;
                if (tag == TAG_TETH_SLIDE) { p.x = p.x + dt * sv.x; p.y = p.y + dt * sv.y; p.z = p.z + dt * sv.z; }
            }
            eng_pos(d, s.pset ^ 1)[i] = p;
            d.vx[i] = vx; d.vy[i] = vy; d.vz[i] = vz;
            m2 = norm2_rn(vx, vy, vz);
        }
        fold_vmax2(d.slots, k, m2);
    }
}

// The record of every recording job (evaluate_macroscopic_properties,
// simulation_record.f90:1205-1314) and its pressure-tensor sample
// (cumulative_pressure, :3151-3205).  Grid (slot, EY).
__global__ void __launch_bounds__(ER) k_e_record(EngDev d)
{
    if (!d.flags->any_record) return;
    const int k = blockIdx.x;
    EngSlot &s = d.slots[k];
    if (!slot_active(s) || !s.record) return;
    double v[RT_N], c[RT_N];
    for (int q = 0; q < RT_N; q++) { v[q] = 0.0; c[q] = 0.0; }
    double pemax = 0.0;
    const int nterm = s.pressure ? RT_N : RT_VSUM + 1;
    int lo, hi;
    job_chunk(s, blockIdx.y, lo, hi);
    for (int i = lo + threadIdx.x; i < hi; i += ER) {
        const double *t = d.rterm + (size_t)i * RT_N;
        for (int q = 0; q < nterm; q++) neumaier(v[q], c[q], t[q]);
        pemax = fmax(pemax, t[RT_PE]);
    }
    __shared__ double smax[ER];
    smax[threadIdx.x] = pemax;
    block_sum<RT_N>(v, c);
    if (threadIdx.x == 0)
        for (int q = 1; q < ER; q++) pemax = fmax(pemax, smax[q]);
    if (!job_merge<RT_N>(d, k, 1, v, c, pemax)) return;
    for (int q = 0; q < RT_N; q++) v[q] = v[q] + c[q];
    const double gnp = (double)s.nmol;
    FmRecord r;
    r.iter = s.iter;
    r.pad_ = 0;
    r.simtime = s.simtime;
    r.vsum = v[RT_VSUM];
    r.mv2sum = v[RT_MV2];
    r.virial = v[RT_VIR];
    r.kinenergy = (0.5 * r.mv2sum) / gnp;
    r.potenergy = (0.5 * v[RT_PE]) / gnp;
    r.totenergy = r.kinenergy + r.potenergy;
    r.temperature = r.mv2sum / (3.0 * gnp);
    r.pressure = (s.density / (gnp * 3.0)) * (r.mv2sum + r.virial / 2.0);
    s.last_rec = r;
    if (s.pressure) {
        const double V = s.volume;
        s.ptensor[0] += v[RT_PXX] / V; s.ptensor[4] += v[RT_PYY] / V; s.ptensor[8] += v[RT_PZZ] / V;
        s.ptensor[1] += v[RT_PXY] / V; s.ptensor[3] += v[RT_PXY] / V;
        s.ptensor[2] += v[RT_PXZ] / V; s.ptensor[6] += v[RT_PXZ] / V;
        s.ptensor[5] += v[RT_PYZ] / V; s.ptensor[7] += v[RT_PYZ] / V;
    }
    s.nsamples += 1;
    if (pemax > 10000.0) slot_fail(&s, ST_PE, s.iter);
}

// ---------------------------------------------------------------------------
// admission / retirement
// ---------------------------------------------------------------------------

__global__ void k_e_scatter_job(EngDev d, int slot, int mol_off, int n, const double *r3, const double *v3,
                                const int32_t *tag, const double *rt3, const double *sv3)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const int i = mol_off + u;
    d.pos0[i] = make_double4(r3[3 * (size_t)u], r3[3 * (size_t)u + 1], r3[3 * (size_t)u + 2], 0.0);
    d.pos1[i] = d.pos0[i];
    d.vx[i] = v3[3 * (size_t)u]; d.vy[i] = v3[3 * (size_t)u + 1]; d.vz[i] = v3[3 * (size_t)u + 2];
    d.ax[i] = 0.0; d.ay[i] = 0.0; d.az[i] = 0.0;
    d.uidx[i] = u;
    d.tag[i] = tag ? tag[u] : TAG_FREE;
    d.rteth[i] = rt3 ? make_double4(rt3[3 * (size_t)u], rt3[3 * (size_t)u + 1], rt3[3 * (size_t)u + 2], 0.0)
                     : make_double4(0, 0, 0, 0);
    d.slidev[i] = sv3 ? make_double4(sv3[3 * (size_t)u], sv3[3 * (size_t)u + 1], sv3[3 * (size_t)u + 2], 0.0)
                      : make_double4(0, 0, 0, 0);
    d.tmv2[i] = 0.0;
    d.nnbr[i] = 0;
    d.slot_of[i] = slot;
}

__global__ void k_e_claim_cells(EngDev d, int slot, int cell_off, int ncell)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    d.cell_slot[cell_off + c] = slot;
    d.cell_count[cell_off + c] = 0;
}

__global__ void k_e_gather_job(EngDev d, int slot, int mol_off, int n, double *r3, double *v3)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const int i = mol_off + a;
    const int u = d.uidx[i];
    const double4 p = eng_pos(d, d.slots[slot].pset)[i];
    r3[3 * (size_t)u] = p.x; r3[3 * (size_t)u + 1] = p.y; r3[3 * (size_t)u + 2] = p.z;
    v3[3 * (size_t)u] = d.vx[i]; v3[3 * (size_t)u + 1] = d.vy[i]; v3[3 * (size_t)u + 2] = d.vz[i];
}

__global__ void k_e_release(EngDev d, int mol_off, int n, int cell_off, int ncell)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) d.slot_of[mol_off + q] = -1;
    if (q < ncell) { d.cell_slot[cell_off + q] = -1; d.cell_count[cell_off + q] = 0; }
}

template <int TPM>
void launch_force_t(const EngDev &d, int mols, bool force_only, cudaStream_t st)
{
    const int g = sgrid((long long)mols * TPM, EF_THREADS, 8);
    if (force_only) {
        if (d.precision == 0) k_e_force<TPM, 0, true, false><<<g, EF_THREADS, 0, st>>>(d);
        else k_e_force<TPM, 1, true, false><<<g, EF_THREADS, 0, st>>>(d);
    } else {
        if (d.precision == 0) {
            k_e_force<TPM, 0, false, false><<<g, EF_THREADS, 0, st>>>(d);
            k_e_force<TPM, 0, false, true><<<g, EF_THREADS, 0, st>>>(d);
        } else {
            k_e_force<TPM, 1, false, false><<<g, EF_THREADS, 0, st>>>(d);
            k_e_force<TPM, 1, false, true><<<g, EF_THREADS, 0, st>>>(d);
        }
    }
}

void launch_force_any(const EngDev &d, int tpm, int mols, bool force_only, cudaStream_t st)
{
    switch (tpm) {
    case 1: launch_force_t<1>(d, mols, force_only, st); break;
    case 2: launch_force_t<2>(d, mols, force_only, st); break;
    case 4: launch_force_t<4>(d, mols, force_only, st); break;
    case 16: launch_force_t<16>(d, mols, force_only, st); break;
    default: launch_force_t<8>(d, mols, force_only, st); break;
    }
}

}  // namespace

int eng_kernels_per_tick() { return 15; }

__global__ void k_e_loop_reset(EngDev d) { d.flags->loop_ticks = 0; }

// Ends an iteration (body_ticks ticks) of the loop: the WHILE node runs
// another while a resident job is set up or running and the launch has run
// fewer than max_ticks ticks, unless a job has failed (the host retires it,
// and re-queues it after a list overflow) or a job is done while queued jobs
// wait for a slot.
__global__ void k_e_continue(EngDev d, int slots, cudaGraphConditionalHandle cond, int body_ticks, int max_ticks)
{
    int live = 0, done = 0, failed = 0;
    for (int k = threadIdx.x; k < slots; k += blockDim.x) {
        const int st = d.slots[k].state;
        live |= st == SLOT_SETUP || st == SLOT_RUN;
        done |= st == SLOT_DONE;
        failed |= st == SLOT_FAILED;
    }
    live = __syncthreads_or(live);
    done = __syncthreads_or(done);
    failed = __syncthreads_or(failed);
    if (threadIdx.x == 0) {
        const int t = d.flags->loop_ticks + body_ticks;
        d.flags->loop_ticks = t;
        const bool to_host = failed || (done && d.flags->queue_waiting);
        cudaGraphSetConditional(cond, (live && !to_host && t < max_ticks) ? 1u : 0u);
    }
}

void eng_loop_reset(const EngDev &d, cudaStream_t st) { k_e_loop_reset<<<1, 1, 0, st>>>(d); }

void eng_loop_continue(const EngDev &d, int slots, cudaGraphConditionalHandle cond, int body_ticks, int max_ticks,
                       cudaStream_t st)
{
    k_e_continue<<<1, 256, 0, st>>>(d, std::min(slots, d.nslots), cond, body_ticks, max_ticks);
}

void eng_tick(const EngDev &d, int tpm, const TickExtent &x, cudaStream_t st)
{
    const int slots = std::min(x.slots, d.nslots);
    const int gm = sgrid(std::min(x.mols, d.mol_cap), 256, 8);
    const int gc = sgrid(std::min(x.cells, d.cell_cap), 256, 8);
    // the slot loops (decision, all-pairs jobs) stop at the extent: every
    // resident slot lies below it, the ones above are empty
    EngDev dx = d;
    dx.nslots = slots;
    k_e_decide<<<1, EDEC, 0, st>>>(dx);
    k_e_wrap_bin<<<gm, 256, 0, st>>>(d);
    k_e_scan<<<slots, ESCAN, 0, st>>>(d);
    k_e_scatter<<<gm, 256, 0, st>>>(d);
    k_e_sort<<<gc, 256, 0, st>>>(d);
    k_e_reorder_gather<<<gm, 256, 0, st>>>(d);
    k_e_reorder_copy<<<gm, 256, 0, st>>>(d);
    // at most one resident wave
    k_e_build<<<sgrid(std::min(x.cells, d.cell_cap), NB_WARPS, 6), NB_THREADS, 0, st>>>(d);
    launch_force_any(d, tpm, std::min(x.mols, d.mol_cap), false, st);
    const dim3 gap(std::min(slots, EAP_XBLOCKS), EAP_YBLOCKS);
    if (d.precision == 0) k_e_force_ap<0><<<gap, EAP_THREADS, 0, st>>>(dx);
    else k_e_force_ap<1><<<gap, EAP_THREADS, 0, st>>>(dx);
    k_e_thermo<<<dim3(slots, EY), ER, 0, st>>>(d);
    k_e_move_lfv<<<gm, 256, 0, st>>>(d);
    k_e_record<<<dim3(slots, EY), ER, 0, st>>>(d);
}

void eng_build_only(const EngDev &d, int cells, cudaStream_t st)
{
    k_e_build<<<sgrid(std::min(cells, d.cell_cap), NB_WARPS, 6), NB_THREADS, 0, st>>>(d);
}

void eng_force_only(const EngDev &d, int tpm, int mols, cudaStream_t st)
{
    launch_force_any(d, tpm, std::min(mols, d.mol_cap), true, st);
}

void eng_scatter_job(const EngDev &d, int slot, int mol_off, int n, const double *r3, const double *v3,
                     const int32_t *tag, const double *rteth3, const double *slidev3, cudaStream_t st)
{
    k_e_scatter_job<<<nblk(n, 256), 256, 0, st>>>(d, slot, mol_off, n, r3, v3, tag, rteth3, slidev3);
}

void eng_claim_cells(const EngDev &d, int slot, int cell_off, int ncell, cudaStream_t st)
{
    if (ncell > 0) k_e_claim_cells<<<nblk(ncell, 256), 256, 0, st>>>(d, slot, cell_off, ncell);
}

void eng_gather_job(const EngDev &d, int slot, int mol_off, int n, double *r3, double *v3, cudaStream_t st)
{
    k_e_gather_job<<<nblk(n, 256), 256, 0, st>>>(d, slot, mol_off, n, r3, v3);
}

void eng_release_job(const EngDev &d, int mol_off, int n, int cell_off, int ncell, cudaStream_t st)
{
    int m = std::max(n, ncell);
    if (m > 0) k_e_release<<<nblk(m, 256), 256, 0, st>>>(d, mol_off, n, cell_off, ncell);
}

}  // namespace fm
