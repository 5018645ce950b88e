// fm_kernels.cu -- sm_100a kernels of the per-timestep MD hot path.
//
// Data layout (device): positions as double4 {x, y, z, 0} so a neighbour
// gather is one 32-byte sector; velocities and accelerations as FP64 SoA for
// coalesced streaming; molecules re-ordered by cell at every rebuild so a
// warp's neighbours share L1 lines.  Distance tests are FP64 without FMA
// contraction (__dmul_rn/__dadd_rn) and periodic images are formed as
// x_src + (+/-)domain, the same two roundings the reference performs when it
// copies a halo molecule (messenger.serial.f90:401, 509) and subtracts
// (linklist.f90:749-750) -- so pair sets match the reference bit for bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>

#include "fm_common.cuh"
#include "fm_device.cuh"
#include "fm_build.cuh"
#include "fm_tile.cuh"

namespace fm {

thread_local bool pdl_capture = false;

namespace {

__device__ __forceinline__ bool frozen(const FmDev &d) { return (d.sc->status & ST_FATAL) != 0u; }

// w of a position: the Mie type (1-based), the Soddemann bead flag (1 for a
// chain bead), or with both the type plus 32 times the flag.
__device__ __forceinline__ int mie_type(double w) { return ((int)w) & 31; }
template <bool MIE>
__device__ __forceinline__ int bead_flag(double w) { return MIE ? ((int)w) >> 5 : (int)w; }

__device__ __forceinline__ void raise_status(const FmDev &d, uint32_t bit, int iter)
{
    if (iter == ITER_DEVICE) iter = d.sc->cur_iter;
    uint32_t old = atomicOr(&d.sc->status, bit);
    if ((old & ST_FATAL) == 0u) d.sc->fail_iter = iter;
}





// Block max of a non-negative double folded into sc->vmax2 (u64 order of
// non-negative doubles equals their numeric order).
__device__ __forceinline__ void block_vmax2(const FmDev &d, double m2)
{
    __shared__ double wmax[32];
    m2 = warp_max(m2);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) wmax[w] = m2;
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        double v = l < nw ? wmax[l] : 0.0;
        v = warp_max(v);
        if (l == 0 && v > 0.0) atomicMax(&d.sc->vmax2, (unsigned long long)__double_as_longlong(v));
    }
}

// ---------------------------------------------------------------------------
// integrator (simulation_move_particles_vv.f90:64-69, 132-135)
// ---------------------------------------------------------------------------

__global__ void k_reset_scalars(FmDev d)
{
    FmScalars *s = d.sc;
    s->rmax = 0.0;
    s->vmax2 = 0ull;
    s->rebuild = 0;
    s->status = 0u;
    s->fail_iter = -1;
    s->max_nbr = 0;
    s->escape_slot = -1;
    s->rebuilds = 0;
    s->digest = 0ull;
    s->digest_n = 0;
    s->nrec_pending = 0;
    s->disp_reset = 1;  // rdisp is allocated as zeros at the first check
    s->dmax = 0ull;
    for (int q = 0; q < 6; q++) s->pacc[q] = 0.0;
    s->pcount = 0;
    s->tile_next = 0;
    s->umax = 0;
}

// r = (r + dt v) + (0.5 dt^2) a ; v = v + (0.5 dt) a   -- pass 1, in place.
__global__ void k_move1(FmDev d)
{
    pdl_enter();
    if (frozen(d)) return;
    double4 *P = cur_pos(d, d.sc->pset);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m2 = 0.0;
    if (i < d.n) {
        double4 p = P[i];
        double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
        double ax = d.ax[i], ay = d.ay[i], az = d.az[i];
        p.x = __dadd_rn(__dadd_rn(p.x, __dmul_rn(d.dt, vx)), __dmul_rn(d.half_dt2, ax));
        p.y = __dadd_rn(__dadd_rn(p.y, __dmul_rn(d.dt, vy)), __dmul_rn(d.half_dt2, ay));
        p.z = __dadd_rn(__dadd_rn(p.z, __dmul_rn(d.dt, vz)), __dmul_rn(d.half_dt2, az));
        vx = __dadd_rn(vx, __dmul_rn(d.half_dt, ax));
        vy = __dadd_rn(vy, __dmul_rn(d.half_dt, ay));
        vz = __dadd_rn(vz, __dmul_rn(d.half_dt, az));
        P[i] = p;
        d.vx[i] = vx; d.vy[i] = vy; d.vz[i] = vz;
        m2 = norm2_rn(vx, vy, vz);
    }
    block_vmax2(d, m2);
}

__global__ void k_move2(FmDev d)
{
    pdl_enter();
    if (frozen(d)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        d.vx[i] = __dadd_rn(d.vx[i], __dmul_rn(d.half_dt, d.ax[i]));
        d.vy[i] = __dadd_rn(d.vy[i], __dmul_rn(d.half_dt, d.ay[i]));
        d.vz[i] = __dadd_rn(d.vz[i], __dmul_rn(d.half_dt, d.az[i]));
    }
}

// simulation_move_particles_lfv NVE (simulation_move_particles_lfv.f90:81-92), in place.
__global__ void k_move_lfv(FmDev d)
{
    pdl_enter();
    if (frozen(d)) return;
    double4 *P = cur_pos(d, d.sc->pset);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m2 = 0.0;
    if (i < d.n) {
        double4 p = P[i];
        double vx = __dadd_rn(d.vx[i], __dmul_rn(d.dt, d.ax[i]));
        double vy = __dadd_rn(d.vy[i], __dmul_rn(d.dt, d.ay[i]));
        double vz = __dadd_rn(d.vz[i], __dmul_rn(d.dt, d.az[i]));
        p.x = __dadd_rn(p.x, __dmul_rn(d.dt, vx));
        p.y = __dadd_rn(p.y, __dmul_rn(d.dt, vy));
        p.z = __dadd_rn(p.z, __dmul_rn(d.dt, vz));
        P[i] = p;
        d.vx[i] = vx; d.vy[i] = vy; d.vz[i] = vz;
        m2 = norm2_rn(vx, vy, vz);
    }
    block_vmax2(d, m2);
}

__global__ void k_vmax(FmDev d)
{
    pdl_enter();
    if (frozen(d)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m2 = 0.0;
    if (i < d.n) m2 = norm2_rn(d.vx[i], d.vy[i], d.vz[i]);
    block_vmax2(d, m2);
}

// Rebuild criterion 2 (simulation_checkrebuild.f90:106-121): rdisp += v dt
// for every molecule (v as the check sees it), and the largest |component|
// into sc->dmax.  After a rebuild the reference deallocates rdisp (:150-152),
// so the next check starts it from zero.
__global__ void k_disp(FmDev d)
{
    pdl_enter();
    if (frozen(d)) return;
    const bool restart = d.sc->disp_reset != 0;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (i < d.n) {
        const double x = __dadd_rn(restart ? 0.0 : d.rdx[i], __dmul_rn(d.vx[i], d.dt));
        const double y = __dadd_rn(restart ? 0.0 : d.rdy[i], __dmul_rn(d.vy[i], d.dt));
        const double z = __dadd_rn(restart ? 0.0 : d.rdz[i], __dmul_rn(d.vz[i], d.dt));
        d.rdx[i] = x; d.rdy[i] = y; d.rdz[i] = z;
        m = fmax(fabs(x), fmax(fabs(y), fabs(z)));
    }
    m = warp_max(m);
    __shared__ double wmax[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) wmax[w] = m;
    __syncthreads();
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double v = l < nw ? wmax[l] : 0.0;
        v = warp_max(v);
        if (l == 0 && v > 0.0) atomicMax(&d.sc->dmax, (unsigned long long)__double_as_longlong(v));
    }
}

// ---------------------------------------------------------------------------
// rebuild decision (simulation_checkrebuild.f90:34, 83-99, 101-103, 106-121, 148-155)
// ---------------------------------------------------------------------------

__device__ __forceinline__ int decide(const FmDev &d, int iter, int flip, int crit, int fixed_rebuild,
                                      double half_min_delta)
{
    FmScalars *s = d.sc;
    if (flip) s->pset ^= 1;
    int rebuild = ((iter + 1) % d.tplot) == 0 ? 1 : 0;
    if (crit == 0) {
        double vmax = sqrt(__longlong_as_double((long long)s->vmax2));
        s->rmax = __dadd_rn(s->rmax, __dmul_rn(vmax, d.dt));
        if (s->rmax > half_min_delta) rebuild = 1;
    } else if (crit == 1) {
        if ((iter % fixed_rebuild) == 0) rebuild = 1;
    } else if (crit == 2) {
        // any(abs(rdisp(:,n)) > 0.5 minval(delta_rneighbr))
        if (__longlong_as_double((long long)s->dmax) > half_min_delta) rebuild = 1;
        s->dmax = 0ull;
        s->disp_reset = rebuild;
    }
    s->vmax2 = 0ull;
    if (rebuild) {
        s->rmax = 0.0;
        s->rebuilds += 1;
    }
    s->rebuild = rebuild;
    return rebuild;
}

__global__ void k_decide(FmDev d, int iter, int flip, int crit, int fixed_rebuild, double half_min_delta)
{
    pdl_enter();
    if (d.sc->status & ST_FATAL) return;
    decide(d, iter, flip, crit, fixed_rebuild, half_min_delta);
}

// The decision as the first node of the rebuild graph (fm_api.cu): the
// iteration comes from the device (g_iter, set by the host at the start of a
// range and advanced here), and the outcome opens the graph's conditional
// body -- the rebuild kernels -- or skips it without launching anything.  A
// frozen state skips it (the handle's default, 0).
__global__ void k_decide_graph(FmDev d, int flip, int crit, int fixed_rebuild, double half_min_delta,
                               cudaGraphConditionalHandle cond, int body_kernels)
{
    FmScalars *s = d.sc;
    const int iter = s->g_iter;
    s->g_iter = iter + 1;
    s->cur_iter = iter;
    if (s->status & ST_FATAL) return;
    const int rebuild = decide(d, iter, flip, crit, fixed_rebuild, half_min_delta);
    if (rebuild) s->graph_kernels += body_kernels;
    cudaGraphSetConditional(cond, rebuild ? 1u : 0u);
}

__global__ void k_set_graph_iter(FmDev d, int iter) { d.sc->g_iter = iter; }

// ---------------------------------------------------------------------------
// cell binning by counting sort (linklist.f90:2645-2679; sendmols wrap
// messenger.serial.f90:961-1028)
// ---------------------------------------------------------------------------

__device__ __forceinline__ bool gate(const FmDev &d, int gated)
{
    if (frozen(d)) return false;
    if (gated && !d.sc->rebuild) return false;
    return true;
}


__global__ void k_wrap_bin(FmDev d, int wrap, int bin, int gated, int iter)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    double4 *P = cur_pos(d, d.sc->pset);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += gridDim.x * blockDim.x) {
        double4 p = P[i];
        if (wrap) {
            double4 q = p;
            if (q.x >= d.hd[0]) q.x = __dsub_rn(q.x, d.L[0]);
            if (q.x < -d.hd[0]) q.x = __dadd_rn(q.x, d.L[0]);
            if (q.y >= d.hd[1]) q.y = __dsub_rn(q.y, d.L[1]);
            if (q.y < -d.hd[1]) q.y = __dadd_rn(q.y, d.L[1]);
            if (q.z >= d.hd[2]) q.z = __dsub_rn(q.z, d.L[2]);
            if (q.z < -d.hd[2]) q.z = __dadd_rn(q.z, d.L[2]);
            if (q.x != p.x || q.y != p.y || q.z != p.z) P[i] = q;
            p = q;
        }
        if (!bin) continue;
        bool bad = false;
        int cx = bin_axis(p.x, d.hd[0], d.cs[0], d.ne[0], bad);
        int cy = bin_axis(p.y, d.hd[1], d.cs[1], d.ne[1], bad);
        int cz = bin_axis(p.z, d.hd[2], d.cs[2], d.ne[2], bad);
        if (bad) {
            raise_status(d, ST_ESCAPE, iter);
            d.sc->escape_slot = i;
        }
        int c = cx + d.ne[0] * (cy + d.ne[1] * cz);
        d.cell_of[i] = c;
        atomicAdd(&d.cell_count[c], 1);
    }
}

// Exclusive scan of the per-cell counts in two parallel passes over tiles of
// SCAN_TILE cells: tile sums, then each tile adds the sum of the tiles before
// it and scans itself.  The counts are zeroed so the scatter can reuse them
// as cursors.
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_PER = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_PER;

__device__ __forceinline__ int block_excl_scan(int v, int *total)
{
    __shared__ int ws[SCAN_THREADS / 32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[w] = incl;
    __syncthreads();
    if (w == 0) {
        int x = lane < SCAN_THREADS / 32 ? ws[lane] : 0, xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += t;
        }
        if (lane < SCAN_THREADS / 32) ws[lane] = xi - x;
        if (lane == SCAN_THREADS / 32 - 1) ws[SCAN_THREADS / 32 - 1] = xi - x, *total = xi;
    }
    __syncthreads();
    return ws[w] + incl - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(FmDev d, int gated)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    __shared__ int tot;
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER;
    int local = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++)
        if (base + k < d.ncell) local += d.cell_count[base + k];
    block_excl_scan(local, &tot);
    if (threadIdx.x == 0) d.tile_sum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(FmDev d, int gated)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    __shared__ int tot, prefix;
    if (threadIdx.x < 32) {
        int acc = 0;
        for (int b = threadIdx.x; b < (int)blockIdx.x; b += 32) acc += d.tile_sum[b];
        acc = warp_sum(acc);
        if (threadIdx.x == 0) prefix = acc;
    }
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER;
    int cnt[SCAN_PER];
    int local = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++) {
        cnt[k] = base + k < d.ncell ? d.cell_count[base + k] : 0;
        local += cnt[k];
    }
    int run = block_excl_scan(local, &tot) + prefix;
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++) {
        if (base + k < d.ncell) {
            d.cell_start[base + k] = run;
            d.cell_count[base + k] = 0;
        }
        run += cnt[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) d.cell_start[d.ncell] = prefix + tot;
}

__global__ void k_scatter(FmDev d, int gated)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += gridDim.x * blockDim.x) {
        int c = d.cell_of[i];
        if (c < 0) continue;  // a subdomain's departed molecule or stale halo copy
        int slot = d.cell_start[c] + atomicAdd(&d.cell_count[c], 1);
        d.perm[slot] = i;
    }
}

// Atomics make the in-cell order arbitrary; sorting each cell by the
// molecules' identity (slot_of: upload index, or global number in a
// subdomain) makes the whole rebuild deterministic and independent of the
// previous order, so that a subdomain lays out a cell's molecules exactly as
// the undivided system does.  One warp per cell: up to 32 members by a
// bitonic sort of (identity, old slot) keys in registers, larger cells by
// lane 0 (insertion sort).
constexpr int SORT_WARPS = 8;
__global__ void __launch_bounds__(32 * SORT_WARPS) k_sort_cells(FmDev d, int gated)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    const int lane = threadIdx.x & 31;
    for (int c = blockIdx.x * SORT_WARPS + (threadIdx.x >> 5); c < d.ncell; c += gridDim.x * SORT_WARPS) {
        const int b = d.cell_start[c], e = d.cell_start[c + 1];
        const int m = e - b;  // uniform across the warp
        if (m <= 32) {
            unsigned long long key = ~0ull;
            if (lane < m) {
                const int o = d.perm[b + lane];
                key = ((unsigned long long)(unsigned)d.slot_of[o] << 32) | (unsigned)o;
            }
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, j);
                    const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
                    key = keep_min ? (key < other ? key : other) : (key > other ? key : other);
                }
            }
            if (lane < m) d.perm[b + lane] = (int)(unsigned)(key & 0xffffffffull);
        } else if (lane == 0) {
            for (int x = b + 1; x < e; x++) {
                const int o = d.perm[x];
                const int key = d.slot_of[o];
                int y = x - 1;
                while (y >= b && d.slot_of[d.perm[y]] > key) {
                    d.perm[y + 1] = d.perm[y];
                    y--;
                }
                d.perm[y + 1] = o;
            }
        }
        if (lane == 0) d.cell_count[c] = 0;  // leave counts zeroed for the next histogram
    }
}

// Gather into scratch in cell order, then copy back, so every array keeps
// its address (the step loop never needs to know whether a rebuild ran).
__global__ void k_reorder_gather(FmDev d, int gated, double4 *tpos, int32_t *tuidx)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    const double4 *P = cur_pos(d, d.sc->pset);
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < d.n; s += gridDim.x * blockDim.x) {
        int o = d.perm[s];
        tpos[s] = P[o];
        d.tvx[s] = d.vx[o]; d.tvy[s] = d.vy[o]; d.tvz[s] = d.vz[o];
        d.tax[s] = d.ax[o]; d.tay[s] = d.ay[o]; d.taz[s] = d.az[o];
        tuidx[s] = d.slot_of[o];
        if (d.potential_flag == 1) {
            d.tchain[s] = d.chain[o]; d.tsubchain[s] = d.subchain[o]; d.tbflag[s] = d.bflag[o];
            if (d.funcy) d.tfuncy[s] = d.funcy[o];
        }
    }
}

__global__ void k_reorder_copy(FmDev d, int gated, const double4 *tpos, const int32_t *tuidx)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    double4 *P = cur_pos(d, d.sc->pset);
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < d.n; s += gridDim.x * blockDim.x) {
        P[s] = tpos[s];
        d.vx[s] = d.tvx[s]; d.vy[s] = d.tvy[s]; d.vz[s] = d.tvz[s];
        d.ax[s] = d.tax[s]; d.ay[s] = d.tay[s]; d.az[s] = d.taz[s];
        d.slot_of[s] = tuidx[s];
        if (d.potential_flag == 1) {
            d.chain[s] = d.tchain[s]; d.subchain[s] = d.tsubchain[s]; d.bflag[s] = d.tbflag[s];
            if (d.funcy) d.funcy[s] = d.tfuncy[s];
        }
    }
}

// ---------------------------------------------------------------------------
// neighbour list from shared-memory cell tiles
// (pair set of assign_to_neighbourlist_halfint_opt, linklist.f90:660-804,
//  1118-1180, stored in both directions)
// ---------------------------------------------------------------------------

// Staging segment table of the tiled force path, one warp per block: the
// exclusive prefix of the block's 128 segment sizes (fm_tile.cuh) and their
// total.  A block whose total exceeds the force kernel's capacity raises
// ST_TILE; the host grows the capacity and builds again.
constexpr int BS_THREADS = 256;
__global__ void __launch_bounds__(BS_THREADS) k_blk_seg(FmDev d, int gated, int iter)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    const int lane = threadIdx.x & 31;
    constexpr int WPB = BS_THREADS / 32;
    int umax = 0;
    for (int blk = blockIdx.x * WPB + (threadIdx.x >> 5); blk < d.tile_nblk; blk += gridDim.x * WPB) {
        const int bx = blk % d.tile_nb[0], by = (blk / d.tile_nb[0]) % d.tile_nb[1];
        const int bz = blk / (d.tile_nb[0] * d.tile_nb[1]);
        int32_t *out = d.blk_off + (size_t)blk * TILE_NSEGP;
        int carry = 0;
#pragma unroll
        for (int h = 0; h < TILE_NSEG / 32; h++) {
            int st, cnt, code;
            tile_segment(d.ne, d.cell_start, 2 * bx, 2 * by, 2 * bz, h * 32 + lane, st, cnt, code);
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            out[h * 32 + lane] = carry + incl - cnt;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) out[TILE_NSEG] = carry;
        umax = max(umax, carry);
    }
    umax = __reduce_max_sync(0xffffffffu, umax);
    if (lane == 0 && umax > 0) {
        atomicMax(&d.sc->umax, umax);
        if (umax > d.tile_ucap) raise_status(d, ST_TILE, iter);
    }
}

// Neighbour rows of every extended cell, one warp per cell or, for sparse
// systems (BLOCKS), per block of 2x2x2 cells (grid-stride); the routines and
// their pair-set argument are in fm_build.cuh.  Both give the same rows.
template <bool POLY, bool BLOCKS, bool TILE>
__global__ void __launch_bounds__(NB_THREADS, 8) k_build_nlist(FmDev d, int gated, int iter)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using Shared = typename std::conditional<BLOCKS, BlockShared<POLY, TILE>, BuildShared<POLY, TILE>>::type;
    // per-warp staging in dynamic shared memory (the largest variants pass 48 KB)
    extern __shared__ __align__(16) unsigned char build_smem[];
    Shared *sh = reinterpret_cast<Shared *>(build_smem);
    CellSys y;
    y.P = cur_pos(d, d.sc->pset);
    y.cell_start = d.cell_start;
    y.mol_off = 0;
    for (int k = 0; k < 3; k++) { y.ne[k] = d.ne[k]; y.cs[k] = d.cs[k]; y.hd[k] = d.hd[k]; y.L[k] = d.L[k]; }
    y.rn2 = d.rn2;
    y.nbr = d.nbr;
    y.nnbr = d.nnbr;
    y.maxn = d.maxn;
    y.max_nbr = &d.sc->max_nbr;
    y.chain = d.chain; y.subchain = d.subchain; y.bflag = d.bflag;
    y.bnd = d.bnd; y.nbond = d.nbond;
    y.nbr16 = d.nbr16; y.maxn16 = d.maxn16; y.tT = d.tile_T; y.tR = d.tile_R; y.blk_off = d.blk_off;
    y.tdummy = d.tile ? tile_boff(d.tile_ucap, d.tile_R) : 0;
    for (int k = 0; k < 3; k++) y.tnb[k] = d.tile_nb[k];
    y.dd = d.dd;
    for (int k = 0; k < 3; k++) y.org[k] = d.dd ? d.org[k] : 0;
    uint32_t over = 0u;
    const int nwork = BLOCKS ? ((d.ne[0] + 1) / 2) * ((d.ne[1] + 1) / 2) * ((d.ne[2] + 1) / 2) : d.ncell;
    // work units handed out NB_CHUNK at a time, so warps that meet empty or
    // halo cells take more: no tail of a few warps with dense cells left
    for (;;) {
        int u0 = 0;
        if (lane == 0) u0 = atomicAdd(&d.sc->build_next, NB_CHUNK);
        u0 = __shfl_sync(0xffffffffu, u0, 0);
        if (u0 >= nwork) break;
        const int u1 = min(u0 + NB_CHUNK, nwork);
        for (int u = u0; u < u1; u++) {
            if constexpr (BLOCKS) over |= build_block<POLY, TILE>(y, u, sh[warp], lane);
            else over |= build_cell<POLY, TILE>(y, u, sh[warp], lane);
        }
    }
    if (lane == 0) {
        if (over & BUILD_OVER_LIST) raise_status(d, ST_NLIST, iter);
        if (over & BUILD_OVER_BONDS) raise_status(d, ST_BOND, iter);
    }
}

// ---------------------------------------------------------------------------
// forces (simulation_compute_forces_LJ_neigbr*, simulation_compute_forces.f90
// :551-726) fused with move(2) and the next move(1)
// ---------------------------------------------------------------------------

constexpr int FORCE_THREADS = 256;

// One pair inside the cutoff: acc (the pair force over rij) accumulated as
// acc * rij, and on record steps the energy and acc * r^2.  PREC bit 0: FP32
// pair magnitude (FP64 rij scales it); bit 1: Mie_potential 1, constants by
// the molecules' types (w of the positions): Mie_accijmag and Mie_energy
// (setup_set_parameters.f90:149-204) with real powers, as s**(lr/2+1).
// Otherwise LJ_accijmag = 48 (s^7 - s^4/2), s = 1/r^2, and LJ_energy
// (:105-135).
template <int PREC, bool REC>
__device__ __forceinline__ double pair_acc(const FmDev &d, double r2, double dx, double dy, double dz, double wi,
                                           double wj, double &fx, double &fy, double &fz, double &pe, double &vir)
{
    constexpr bool F32 = (PREC & 1) != 0, MIE = (PREC & 2) != 0, SOD = (PREC & 4) != 0;
    if (SOD) {
        // simulation_compute_forces_Soddemann_neigbr_halfint (:793-888): WCA
        // inside wca_cut2, the cosine well eps a s^2 sin(a s + b) beyond it
        // (the reference's expression, s = 1/r^2); no potshift.  The WCA force
        // is get_accijmag: Mie_accijmag of the pair's types with
        // Mie_potential 1, its energy the LJ-WCA expression either way.
        const double eps = d.sod_eps[bead_flag<MIE>(wi) + bead_flag<MIE>(wj)];
        const bool wca = r2 < SOD_WCA_CUT2;
        if (!F32) {
            const double s = __drcp_rn(r2);
            const double s2 = s * s;
            double acc;
            if (wca && MIE) {
                const FmMiePair &m = d.mie_pair[(mie_type(wi) - 1) + MIE_MAXT * (mie_type(wj) - 1)];
                acc = m.ceps * (m.lr * pow(s, m.er1) - m.ala * pow(s, m.ea1));
            } else if (wca) {
                const double s4 = s2 * s2;
                acc = 48.0 * (s4 * s2 * s - 0.5 * s4);  // get_accijmag = LJ_accijmag
            } else {
                acc = (eps * SOD_A * s2) * sin(s * SOD_A + SOD_B);
            }
            fx += acc * dx; fy += acc * dy; fz += acc * dz;
            if (REC) {
                if (wca) {
                    const double s3 = s2 * s, s6 = s3 * s3;
                    pe += 4.0 * (s6 - s3 + 0.25) - eps;
                } else {
                    pe += 0.5 * eps * (cos(SOD_A * r2 + SOD_B) - 1.0);
                }
                vir += acc * r2;
            }
        } else {
            const float s = rcp_f32((float)r2);
            const float s2 = s * s;
            float accf;
            if (wca && MIE) {
                const FmMiePair &m = d.mie_pair[(mie_type(wi) - 1) + MIE_MAXT * (mie_type(wj) - 1)];
                accf = (float)m.ceps * ((float)m.lr * powf(s, (float)m.er1) - (float)m.ala * powf(s, (float)m.ea1));
            } else if (wca) {
                const float s4 = s2 * s2;
                accf = 48.0f * (s4 * s2 * s - 0.5f * s4);
            } else {
                accf = ((float)eps * (float)SOD_A * s2) * sinf(s * (float)SOD_A + (float)SOD_B);
            }
            const double acc = (double)accf;
            fx = fma(acc, dx, fx); fy = fma(acc, dy, fy); fz = fma(acc, dz, fz);
            if (REC) {
                if (wca) {
                    const float s3 = s2 * s, s6 = s3 * s3;
                    pe += (double)(4.0f * (s6 - s3 + 0.25f)) - eps;
                } else {
                    pe += (double)(0.5f * (float)eps * (cosf((float)SOD_A * (float)r2 + (float)SOD_B) - 1.0f));
                }
                vir += acc * r2;
            }
        }
        return 0.0;  // the Soddemann routine records no pressure-tensor term
    }
    if (MIE) {
        const FmMiePair &m = d.mie_pair[(mie_type(wi) - 1) + MIE_MAXT * (mie_type(wj) - 1)];
        if (!F32) {
            const double s = __drcp_rn(r2);  // == 1.0 / r2
            const double acc = m.ceps * (m.lr * pow(s, m.er1) - m.ala * pow(s, m.ea1));
            fx += acc * dx; fy += acc * dy; fz += acc * dz;
            if (REC) {
                pe += m.ceps * (pow(s, m.er) - m.alpha * pow(s, m.ea)) - m.shift;
                vir += acc * r2;
            }
            return acc;
        } else {
            const float s = rcp_f32((float)r2);
            const double acc = (double)((float)m.ceps * ((float)m.lr * powf(s, (float)m.er1) -
                                                         (float)m.ala * powf(s, (float)m.ea1)));
            fx = fma(acc, dx, fx); fy = fma(acc, dy, fy); fz = fma(acc, dz, fz);
            if (REC) {
                pe += (double)((float)m.ceps * (powf(s, (float)m.er) - (float)m.alpha * powf(s, (float)m.ea))) - m.shift;
                vir += acc * r2;
            }
            return acc;
        }
    } else if (!F32) {
        const double s = __drcp_rn(r2);  // == 1.0 / r2 (both correctly rounded)
        const double s2 = s * s, s4 = s2 * s2;
        const double acc = 48.0 * (s4 * s2 * s - 0.5 * s4);
        fx += acc * dx; fy += acc * dy; fz += acc * dz;
        if (REC) {
            const double s3 = s2 * s, s6 = s3 * s3;
            pe += 4.0 * (s6 - s3) - d.potshift;  // LJ_energy (:126-135)
            vir += acc * r2;
        }
        return acc;
    } else {
        // FP32 pair magnitude; the FP64 rij scales it (one conversion)
        const float s = rcp_f32((float)r2);
        const float s2 = s * s, s4 = s2 * s2;
        const double acc = (double)(48.0f * (s4 * s2 * s - 0.5f * s4));
        fx = fma(acc, dx, fx); fy = fma(acc, dy, fy); fz = fma(acc, dz, fz);
        if (REC) {
            const float s3 = s2 * s, s6 = s3 * s3;
            pe += (double)(4.0f * (s6 - s3)) - d.potshift;
            vir += acc * r2;
        }
        return acc;
    }
}

// pressure_tensor_forces (simulation_record.f90:6239-6256): rf += acc rij rij,
// the six distinct components xx yy zz xy xz yz.
__device__ __forceinline__ void add_rf(double (&rf)[6], double acc, double dx, double dy, double dz)
{
    const double ax = acc * dx, ay = acc * dy, az = acc * dz;
    rf[0] += ax * dx; rf[1] += ay * dy; rf[2] += az * dz;
    rf[3] += ax * dy; rf[4] += ax * dz; rf[5] += ay * dz;
}

// Record-step pressure terms of one molecule: v v + rf/2 (cumulative_pressure
// case 1, simulation_record.f90:3170-3199; no mass factor there).
__device__ __forceinline__ void pressure_part(double (&part)[RS_N], double wx, double wy, double wz,
                                              const double (&rf)[6])
{
    part[RS_PXX] = wx * wx + rf[0] / 2.0; part[RS_PYY] = wy * wy + rf[1] / 2.0;
    part[RS_PZZ] = wz * wz + rf[2] / 2.0; part[RS_PXY] = wx * wy + rf[3] / 2.0;
    part[RS_PXZ] = wx * wz + rf[4] / 2.0; part[RS_PYZ] = wy * wz + rf[5] / 2.0;
}

// Integrator epilogue of molecule i with its summed LJ force: stores a (and PE
// and virial on record steps) and, by MODE,
//   1  move(2)                               (simulation_move_particles_vv.f90:132-135)
//   2  move(2) + move(1) of the next step    (:64-69), new positions into pset^1
//   3  leap-frog v += dt a, r += dt v        (simulation_move_particles_lfv.f90:81-92)
// The record partials use v after move(2) for velocity Verlet and v + a dt/2
// for leap-frog (simulation_record.f90:1236-1252).  Returns |v|^2 after a
// position update (modes 2, 3), else 0.
// DIV false: the forces are accelerations already (the Soddemann pairs and
// the mass-divided bonds of a Mie + Soddemann system); the kinetic terms are
// still mass-weighted.
template <bool REC, int MODE, bool MIE = false, bool DIV = true>
__device__ __forceinline__ double epilogue(const FmDev &d, int pset, int i, double4 p, double fx, double fy,
                                           double fz, double pe, double vir, double (&part)[RS_N],
                                           const double (&rf)[6])
{
    if (REC && d.pressure) {  // kept for a record taken after the move (fm_evaluate_macroscopic_properties)
        double *q = d.rf6 + 6 * (size_t)i;
#pragma unroll
        for (int k = 0; k < 6; k++) q[k] = rf[k];
    }
    double mass = 1.0;  // LJ_mass; Mie_mass = mass_lookup(moltype)
    if (MIE) {
        mass = d.mie_mass[mie_type(p.w) - 1];
        if (DIV) { fx = fx / mass; fy = fy / mass; fz = fz / mass; }
    }
    d.ax[i] = fx; d.ay[i] = fy; d.az[i] = fz;
    if (REC) { d.pe[i] = pe; d.vir[i] = vir; }
    double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
    double m2 = 0.0;
    if (MODE == 3) {
        if (REC) {
            const double wx = __dadd_rn(vx, __dmul_rn(__dmul_rn(0.5, fx), d.dt));
            const double wy = __dadd_rn(vy, __dmul_rn(__dmul_rn(0.5, fy), d.dt));
            const double wz = __dadd_rn(vz, __dmul_rn(__dmul_rn(0.5, fz), d.dt));
            part[RS_PE] = pe; part[RS_VIR] = vir; part[RS_PEMAX] = pe;
            part[RS_MV2] = MIE ? mass * norm2_rn(wx, wy, wz) : norm2_rn(wx, wy, wz);
            part[RS_VSUM] = MIE ? mass * __dadd_rn(__dadd_rn(wx, wy), wz) : __dadd_rn(__dadd_rn(wx, wy), wz);
            if (d.pressure) pressure_part(part, wx, wy, wz, rf);
        }
        vx = __dadd_rn(vx, __dmul_rn(d.dt, fx));
        vy = __dadd_rn(vy, __dmul_rn(d.dt, fy));
        vz = __dadd_rn(vz, __dmul_rn(d.dt, fz));
        p.x = __dadd_rn(p.x, __dmul_rn(d.dt, vx));
        p.y = __dadd_rn(p.y, __dmul_rn(d.dt, vy));
        p.z = __dadd_rn(p.z, __dmul_rn(d.dt, vz));
        cur_pos(d, pset ^ 1)[i] = p;
        d.vx[i] = vx; d.vy[i] = vy; d.vz[i] = vz;
        return norm2_rn(vx, vy, vz);
    }
    if (MODE >= 1) {
        vx = __dadd_rn(vx, __dmul_rn(d.half_dt, fx));
        vy = __dadd_rn(vy, __dmul_rn(d.half_dt, fy));
        vz = __dadd_rn(vz, __dmul_rn(d.half_dt, fz));
    }
    if (REC) {
        double wx = vx, wy = vy, wz = vz;
        if (MODE == 0 && d.integrator == 0) {  // forces only, leap-frog record velocity
            wx = __dadd_rn(vx, __dmul_rn(__dmul_rn(0.5, fx), d.dt));
            wy = __dadd_rn(vy, __dmul_rn(__dmul_rn(0.5, fy), d.dt));
            wz = __dadd_rn(vz, __dmul_rn(__dmul_rn(0.5, fz), d.dt));
        }
        part[RS_PE] = pe; part[RS_VIR] = vir; part[RS_PEMAX] = pe;
        part[RS_MV2] = MIE ? mass * norm2_rn(wx, wy, wz) : norm2_rn(wx, wy, wz);
        part[RS_VSUM] = MIE ? mass * __dadd_rn(__dadd_rn(wx, wy), wz) : __dadd_rn(__dadd_rn(wx, wy), wz);
        if (d.pressure) pressure_part(part, wx, wy, wz, rf);
    }
    if (MODE == 2) {
        p.x = __dadd_rn(__dadd_rn(p.x, __dmul_rn(d.dt, vx)), __dmul_rn(d.half_dt2, fx));
        p.y = __dadd_rn(__dadd_rn(p.y, __dmul_rn(d.dt, vy)), __dmul_rn(d.half_dt2, fy));
        p.z = __dadd_rn(__dadd_rn(p.z, __dmul_rn(d.dt, vz)), __dmul_rn(d.half_dt2, fz));
        vx = __dadd_rn(vx, __dmul_rn(d.half_dt, fx));
        vy = __dadd_rn(vy, __dmul_rn(d.half_dt, fy));
        vz = __dadd_rn(vz, __dmul_rn(d.half_dt, fz));
        cur_pos(d, pset ^ 1)[i] = p;
        m2 = norm2_rn(vx, vy, vz);
    }
    if (MODE >= 1) { d.vx[i] = vx; d.vy[i] = vy; d.vz[i] = vz; }
    return m2;
}

// FENE springs of molecule i (simulation_compute_forces_poly,
// simulation_compute_forces.f90:731-789): accijmag = -k/(1 - r^2/R0^2)
// (FENE_accijmag, setup_set_parameters.f90:348-358), energy
// 0.5 k R0^2 log(1 - r^2/R0^2) (:371-380), in FP64 for every precision form.
// A bond at or beyond R0 is the reference's polymer_bond_error.
template <bool REC, bool MIE>
__device__ __forceinline__ void fene_bonds(const FmDev &d, const double4 *P, int i, double &fx, double &fy,
                                           double &fz, double &pe, double &vir, double (&rf)[6])
{
    const double4 pi = P[i];
    const int nb = d.nbond[i];
    for (int b = 0; b < nb; b++) {
        const int e = d.bnd[(size_t)i * 4 + b];
        const int code = e >> NB_SHIFT_BITS;
        const double4 pj = P[e & NB_INDEX_MASK];
        const double xj = (code & 3) != 1 ? __dadd_rn(pj.x, (code & 3) == 2 ? d.L[0] : -d.L[0]) : pj.x;
        const double yj = ((code >> 2) & 3) != 1 ? __dadd_rn(pj.y, ((code >> 2) & 3) == 2 ? d.L[1] : -d.L[1]) : pj.y;
        const double zj = ((code >> 4) & 3) != 1 ? __dadd_rn(pj.z, ((code >> 4) & 3) == 2 ? d.L[2] : -d.L[2]) : pj.z;
        const double dx = __dsub_rn(pi.x, xj), dy = __dsub_rn(pi.y, yj), dz = __dsub_rn(pi.z, zj);
        const double r2 = norm2_rn(dx, dy, dz);
        if (MIE) {
            // harmonic_accijmag / harmonic_energy (setup_set_parameters.f90:384-437):
            // -k (|r| - r0)/|r| and k/2 (|r| - r0)^2, constants by type pair
            const FmMiePair &m = d.mie_pair[(mie_type(pi.w) - 1) + MIE_MAXT * (mie_type(pj.w) - 1)];
            const double rm = sqrt(r2), dr = rm - m.r0;
            const double acc = -m.k * dr / rm;
            fx += acc * dx; fy += acc * dy; fz += acc * dz;
            if (REC) {
                pe += 0.5 * m.k * (dr * dr);
                vir += acc * r2;
                if (d.pressure) add_rf(rf, acc, dx, dy, dz);  // :768-770
            }
            continue;
        }
        if (r2 >= d.R0_2) {
            uint32_t old = atomicOr(&d.sc->status, ST_BOND);
            if ((old & ST_FATAL) == 0u) d.sc->fail_iter = -2;
            continue;
        }
        const double q = r2 / d.R0_2;
        const double acc = -d.k_c / (1.0 - q);
        fx += acc * dx; fy += acc * dy; fz += acc * dz;
        if (REC) {
            pe += 0.5 * d.k_c * d.R0 * d.R0 * log(1.0 - q);
            vir += acc * r2;
            if (d.pressure) add_rf(rf, acc, dx, dy, dz);  // :768-770
        }
    }
}

// ---------------------------------------------------------------------------
// angular_potential (simulation_compute_forces_angular,
// simulation_compute_forces.f90:981-1048; angular_harmonic_force,
// setup_set_parameters.f90:441-489)
// ---------------------------------------------------------------------------

// The reference's triple of middle bead j: i = its first bond, k = its second
// (in discovery order), rij = r_i - r_j, rjk = r_j - r_k with the partners'
// periodic images (x_src +/- L, one rounding), theta = acos(rij.rjk /
// (|rij| |rjk|)) and
//   aForce(1) = -(k (theta - theta_0) / (|rij| sin theta)) (rjk/|rjk| - rij/|rij| cos theta)
//   aForce(3) = -(k (theta - theta_0) / (|rjk| sin theta)) (rij/|rij| - rjk/|rjk| cos theta)
//   aForce(2) = -aForce(1) - aForce(3)   (all zero when theta < 1e-5);
// the reference then subtracts aForce(1), (2), (3) from the forces on i, j,
// k.  Every molecule evaluates the triples it belongs to in the middle
// bead's frame, so the three see the same numbers.  k_ijk < 1e-5 leaves the
// reference's result unset: ST_ANGLE.
__device__ __forceinline__ bool angular_triple(const FmDev &d, const double4 *P, int j, double (&f1)[3],
                                               double (&f3)[3])
{
    const int e0 = d.bnd[(size_t)j * 4], e1 = d.bnd[(size_t)j * 4 + 1];
    const double4 pj = P[j], pi = P[e0 & NB_INDEX_MASK], pk = P[e1 & NB_INDEX_MASK];
    const int c0 = e0 >> NB_SHIFT_BITS, c1 = e1 >> NB_SHIFT_BITS;
    const double ri[3] = {image(pi.x, (c0 & 3) - 1, d.L[0]), image(pi.y, ((c0 >> 2) & 3) - 1, d.L[1]),
                          image(pi.z, ((c0 >> 4) & 3) - 1, d.L[2])};
    const double rk[3] = {image(pk.x, (c1 & 3) - 1, d.L[0]), image(pk.y, ((c1 >> 2) & 3) - 1, d.L[1]),
                          image(pk.z, ((c1 >> 4) & 3) - 1, d.L[2])};
    const double rj[3] = {pj.x, pj.y, pj.z};
    const int nt = d.ang_nt;
    const int q = (mie_type(pi.w) - 1) + nt * ((mie_type(pj.w) - 1) + nt * (mie_type(pk.w) - 1));
    const double kk = d.ang_k[q], t0 = d.ang_t0[q];
    f1[0] = f1[1] = f1[2] = 0.0;
    f3[0] = f3[1] = f3[2] = 0.0;
    if (kk < 1e-5) return false;
    double rij[3], rjk[3];
#pragma unroll
    for (int c = 0; c < 3; c++) { rij[c] = __dsub_rn(ri[c], rj[c]); rjk[c] = __dsub_rn(rj[c], rk[c]); }
    const double mij = sqrt(norm2_rn(rij[0], rij[1], rij[2]));
    const double mjk = sqrt(norm2_rn(rjk[0], rjk[1], rjk[2]));
    const double dot = __dadd_rn(__dadd_rn(__dmul_rn(rij[0], rjk[0]), __dmul_rn(rij[1], rjk[1])),
                                 __dmul_rn(rij[2], rjk[2]));
    const double th = acos(dot / (mij * mjk));
    if (th < 1e-5) return true;
    const double ct = cos(th), stt = sin(th);
    const double a1 = kk * (th - t0) / (mij * stt), a3 = kk * (th - t0) / (mjk * stt);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        f1[c] = -a1 * (rjk[c] / mjk - rij[c] / mij * ct);
        f3[c] = -a3 * (rij[c] / mij - rjk[c] / mjk * ct);
    }
    return true;
}

// The angular forces on molecule m (added to its force sum before the
// division by its mass): -aForce(2) of its own triple when it is a middle
// bead, and -aForce(1) or -aForce(3) of each bonded middle bead's triple in
// which it is the bead i or k.
__device__ __forceinline__ void angular_forces(const FmDev &d, const double4 *P, int m, double &fx, double &fy,
                                               double &fz)
{
    double f1[3], f3[3];
    bool ok = true;
    if (d.funcy[m] == 2) {
        ok &= angular_triple(d, P, m, f1, f3);
        fx += f1[0] + f3[0]; fy += f1[1] + f3[1]; fz += f1[2] + f3[2];  // -aForce(2)
    }
    const int nb = d.nbond[m];
    for (int b = 0; b < nb; b++) {
        const int e = d.bnd[(size_t)m * 4 + b];
        const int p = e & NB_INDEX_MASK;
        if (d.funcy[p] != 2) continue;
        const int c = e >> NB_SHIFT_BITS;  // m as p sees it: the opposite image
        const int back = m | (((2 - (c & 3)) | ((2 - ((c >> 2) & 3)) << 2) | ((2 - ((c >> 4) & 3)) << 4))
                              << NB_SHIFT_BITS);
        ok &= angular_triple(d, P, p, f1, f3);
        if (d.bnd[(size_t)p * 4] == back) { fx -= f1[0]; fy -= f1[1]; fz -= f1[2]; }
        else if (d.bnd[(size_t)p * 4 + 1] == back) { fx -= f3[0]; fy -= f3[1]; fz -= f3[2]; }
        else ok = false;
    }
    if (!ok) {
        uint32_t old = atomicOr(&d.sc->status, ST_ANGLE);
        if ((old & ST_FATAL) == 0u) d.sc->fail_iter = -3;
    }
}

// Discovery key of the bond (j, entry) in the reference's list build
// (assign_to_neighbourlist_halfint_opt, linklist.f90:660-804, where
// check_update_adjacentbeadinfo appends each bonded pair to both rows as it is
// met): interior cells in (x, y, z) loop order with z fastest; in each cell
// first the in-cell pairs (list order, the later member after the earlier),
// then the 13 forward shifts (shift, owner, partner); the cells' lists are in
// decreasing molecule number (head insertion, assign_to_cell loops 1..np).
// A pair across the periodic boundary is met only in the halo sweeps that
// follow (:778-802): after every interior pair, ordered here by the partner's
// molecule number.
__device__ int ang_cell_of(const FmDev &d, int s)
{
    int lo = 0, hi = d.ncell - 1;  // largest c with cell_start[c] <= s
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (d.cell_start[mid] <= s) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ int ang_list_pos(const FmDev &d, int c, int s)
{
    const int me = d.slot_of[s];
    int pos = 0;
    for (int t = d.cell_start[c]; t < d.cell_start[c + 1]; t++) pos += d.slot_of[t] > me ? 1 : 0;
    return pos;
}
__device__ unsigned long long ang_key(const FmDev &d, int j, int e)
{
    const int p = e & NB_INDEX_MASK, code = e >> NB_SHIFT_BITS;
    if (code != NB_NOSHIFT) return (1ull << 62) | (unsigned long long)d.slot_of[p];
    const int SX[13] = {1, 1, 0, -1, 0, 1, 1, 0, -1, -1, -1, 0, 1};  // the 13 forward shifts (:686-688)
    const int SY[13] = {0, 1, 1, 1, 0, 0, 1, 1, 1, 0, -1, -1, -1};
    const int SZ[13] = {0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1};
    const int cj = ang_cell_of(d, j), cp = ang_cell_of(d, p);
    const int ne0 = d.ne[0], ne1 = d.ne[1];
    const int jx = cj % ne0, jy = (cj / ne0) % ne1, jz = cj / (ne0 * ne1);
    const int px = cp % ne0, py = (cp / ne0) % ne1, pz = cp / (ne0 * ne1);
    const int pj = ang_list_pos(d, cj, j), pp = ang_list_pos(d, cp, p);
    int oc = cj, sub = 0, pa = min(pj, pp), pb = max(pj, pp);
    if (cj != cp) {
        const int dx = px - jx, dy = py - jy, dz = pz - jz;
        for (int k = 0; k < 13; k++) {
            if (SX[k] == dx && SY[k] == dy && SZ[k] == dz) { oc = cj; sub = 1 + k; pa = pj; pb = pp; }
            if (SX[k] == -dx && SY[k] == -dy && SZ[k] == -dz) { oc = cp; sub = 1 + k; pa = pp; pb = pj; }
        }
    }
    const int ox = oc % ne0, oy = (oc / ne0) % ne1, oz = oc / (ne0 * ne1);
    const unsigned long long rank = ((unsigned long long)(ox - 1) * (unsigned)(d.nc[1]) + (unsigned)(oy - 1)) *
                                        (unsigned)(d.nc[2]) + (unsigned)(oz - 1);
    return (rank << 34) | ((unsigned long long)sub << 30) | ((unsigned long long)pa << 15) | (unsigned long long)pb;
}

__global__ void k_angular_order(FmDev d, int gated, int iter)
{
    pdl_enter();
    if (!gate(d, gated)) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
        if (d.funcy[j] != 2) continue;
        if (d.nbond[j] != 2) { raise_status(d, ST_ANGLE, iter); continue; }
        const int e0 = d.bnd[(size_t)j * 4], e1 = d.bnd[(size_t)j * 4 + 1];
        if (ang_key(d, j, e1) < ang_key(d, j, e0)) {
            d.bnd[(size_t)j * 4] = e1;
            d.bnd[(size_t)j * 4 + 1] = e0;
        }
    }
}

__global__ void k_set_funcy(FmDev d, const int32_t *funcy_up)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < d.n) d.funcy[u] = funcy_up[u];  // slots still equal upload indices
}

// (s, c) += (s2, c2): Neumaier merge of two compensated partial sums.
__device__ __forceinline__ void nmerge(double &s, double &c, double s2, double c2)
{
    neumaier(s, c, s2);
    c += c2;
}

// Block reduction of the record partials into row `row` of d.partial:
// Neumaier-compensated sums in a fixed tree order (warp xor tree, then the
// warps in index order), the row holding the compensated value rounded once;
// PE max for the PE check.
template <int NT = FORCE_THREADS>
__device__ __forceinline__ void block_partials(const FmDev &d, double v[RS_N], int row)
{
    __shared__ double ws[RS_N][NT / 32], wc[RS_N][NT / 32];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < RS_N; k++) {
        double x = v[k], c = 0.0;
        if (k == RS_PEMAX) {
            x = warp_max(x);
        } else {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double x2 = __shfl_xor_sync(0xffffffffu, x, o), c2 = __shfl_xor_sync(0xffffffffu, c, o);
                nmerge(x, c, x2, c2);
            }
        }
        if (l == 0) { ws[k][w] = x; wc[k][w] = c; }
    }
    __syncthreads();
    if (threadIdx.x < RS_N) {
        int k = threadIdx.x;
        double acc = ws[k][0], cmp = wc[k][0];
        for (int q = 1; q < NT / 32; q++) {
            if (k == RS_PEMAX) acc = fmax(acc, ws[k][q]);
            else nmerge(acc, cmp, ws[k][q], wc[k][q]);
        }
        d.partial[(size_t)row * RS_N + k] = k == RS_PEMAX ? acc : acc + cmp;
    }
}

// Pair sum of molecule i over its list row: lane `lane` of the molecule's
// TPM lanes takes 4 consecutive entries per iteration (one 16-byte load) and
// issues their 4 gathers before any arithmetic.  Entries without an image
// shift (all but the rows of boundary cells) skip the shift decoding.
template <int TPM, bool REC, int PREC>
__device__ __forceinline__ void list_pairs(const FmDev &d, const double4 *__restrict__ P, int i, int lane,
                                           const double4 &pi, double &fx, double &fy, double &fz, double &pe,
                                           double &vir, double (&rf)[6])
{
    const int cnt = d.nnbr[i];
    const int32_t *__restrict__ L = d.nbr + nb_row(i, d.maxn);  // entries k0..k0+3 at L + nb_col(k0) (16-byte aligned)
    const double Lx = d.L[0], Ly = d.L[1], Lz = d.L[2];
    const double rc2 = d.rc2;
    for (int k0 = lane * 4; k0 < cnt; k0 += 4 * TPM) {
        const int4 e4 = ld_stream_int4(reinterpret_cast<const int4 *>(L + nb_col(k0)));
        const int ev[4] = {e4.x, e4.y, e4.z, e4.w};
        double4 pj[4];
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (k0 + q < cnt) pj[q] = ldg_pos(P + (ev[q] & NB_INDEX_MASK));
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (k0 + q >= cnt) break;
            const int code = ev[q] >> NB_SHIFT_BITS;
            double xj = pj[q].x, yj = pj[q].y, zj = pj[q].z;
            if (code != NB_NOSHIFT) {
                const int ssx = (code & 3) - 1, ssy = ((code >> 2) & 3) - 1, ssz = ((code >> 4) & 3) - 1;
                xj = ssx ? __dadd_rn(xj, ssx > 0 ? Lx : -Lx) : xj;
                yj = ssy ? __dadd_rn(yj, ssy > 0 ? Ly : -Ly) : yj;
                zj = ssz ? __dadd_rn(zj, ssz > 0 ? Lz : -Lz) : zj;
            }
            const double dx = __dsub_rn(pi.x, xj);
            const double dy = __dsub_rn(pi.y, yj);
            const double dz = __dsub_rn(pi.z, zj);
            const double r2 = norm2_rn(dx, dy, dz);
            if (r2 < rc2) {
                const double acc = pair_acc<PREC, REC>(d, r2, dx, dy, dz, pi.w, pj[q].w, fx, fy, fz, pe, vir);
                // every partner of i in the full list: the half list's i and j sides
                if (REC && d.pressure) add_rf(rf, acc, dx, dy, dz);
            }
        }
    }
}

// Bonded terms and the integrator epilogue of molecule i once its pair sum is
// complete; returns |v|^2 after a position update (epilogue()).
template <bool REC, int MODE, int PREC>
__device__ __forceinline__ double owner_finish(const FmDev &d, int pset, const double4 *__restrict__ P, int i,
                                               double fx, double fy, double fz, double pe, double vir,
                                               double (&part)[RS_N], double (&rf)[6])
{
    if constexpr ((PREC & 6) == 6) {
        // Mie + Soddemann: the Soddemann pairs are not divided by a mass
        // (:852-860), the bonds of simulation_compute_forces_poly are
        // (:752-754)
        const double4 pi = P[i];
        double bx = 0.0, by = 0.0, bz = 0.0;
        if (d.potential_flag == 1) fene_bonds<REC, true>(d, P, i, bx, by, bz, pe, vir, rf);
        const double mass = d.mie_mass[mie_type(pi.w) - 1];
        fx += bx / mass; fy += by / mass; fz += bz / mass;
        return epilogue<REC, MODE, true, false>(d, pset, i, pi, fx, fy, fz, pe, vir, part, rf);
    } else {
        if (d.potential_flag == 1) fene_bonds<REC, (PREC & 2) != 0>(d, P, i, fx, fy, fz, pe, vir, rf);
        if constexpr ((PREC & 2) != 0) {  // angular_potential needs the Mie types
            if (d.angular) angular_forces(d, P, i, fx, fy, fz);
        }
        // a(:,i) = sum acc rij / mass (LJ_mass = 1; Mie_mass by type)
        return epilogue<REC, MODE, (PREC & 2) != 0>(d, pset, i, P[i], fx, fy, fz, pe, vir, part, rf);
    }
}

template <int TPM, bool REC, int MODE, int PREC>
__global__ void __launch_bounds__(FORCE_THREADS) k_force(FmDev d)
{
    pdl_enter();
    if (frozen(d)) return;
    const int pset = d.sc->pset;
    const double4 *__restrict__ P = cur_pos(d, pset);
    const int gt = blockIdx.x * FORCE_THREADS + threadIdx.x;
    const int i = gt / TPM;
    const int lane = gt % TPM;
    const bool active = i < d.n;
    double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0, vir = 0.0;
    double rf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (active) list_pairs<TPM, REC, PREC>(d, P, i, lane, P[i], fx, fy, fz, pe, vir, rf);
    if (TPM > 1) {
#pragma unroll
        for (int o = TPM / 2; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
            if (REC) {
                pe += __shfl_xor_sync(0xffffffffu, pe, o);
                vir += __shfl_xor_sync(0xffffffffu, vir, o);
                if (d.pressure) {
#pragma unroll
                    for (int k = 0; k < 6; k++) rf[k] += __shfl_xor_sync(0xffffffffu, rf[k], o);
                }
            }
        }
    }
    double part[RS_N] = {};
    double m2 = 0.0;
    if (active && lane == 0) m2 = owner_finish<REC, MODE, PREC>(d, pset, P, i, fx, fy, fz, pe, vir, part, rf);
    if (REC) block_partials(d, part, blockIdx.x);
    if (MODE >= 2) block_vmax2(d, m2);
}

// ---------------------------------------------------------------------------
// tiled forces: the same pair sums, partners read from a shared-memory
// staging of the block's neighbourhood (fm_tile.cuh) instead of gathered
// from global memory one list entry at a time
// ---------------------------------------------------------------------------

// One CTA takes a block of 2x2x2 cells at a time (handed out from an atomic
// counter): it stages the positions of the block's 4x4x4-cell neighbourhood,
// periodic images applied with the same single FP64 add as every other path
// (image(): x_src +/- L), as FP64 rows of 32 candidates; then T lanes per
// owner walk the owner's row of 16-bit staging offsets, T consecutive entries
// at a time, and evaluate each pair exactly as k_force does (FP64 cutoff test
// without contraction, the same pair_acc and epilogue).  Record partials are
// written per block (a fixed row whatever CTA took it), so the record sums do
// not depend on the hand-out order.
constexpr int FT_THREADS = FORCE_THREADS;
constexpr int FT_WARPS = FT_THREADS / 32;

// FP32 LJ pair of the precision form on the tiled path: the pair magnitude
// 48 s^7 - 24 s^4 = s^4 (48 s^3 - 24) in FP32 from an approximate reciprocal
// (rcp.approx, relative error ~2^-23 -- far inside the form's 1e-5
// tolerance), scaled by the FP64 rij; LJ_energy 4 (s^6 - s^3) - potshift on
// record steps.
template <bool REC>
__device__ __forceinline__ double lj32_pair(double r2, double dx, double dy, double dz, double potshift,
                                            double &fx, double &fy, double &fz, double &pe, double &vir)
{
    const float r2f = __double2float_rn(r2);
    float s;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(r2f));
    const float s2 = s * s, s3 = s2 * s, s4 = s2 * s2;
    const double acc = (double)(s4 * fmaf(48.0f, s3, -24.0f));
    fx = fma(acc, dx, fx); fy = fma(acc, dy, fy); fz = fma(acc, dz, fz);
    if (REC) {
        pe += (double)(4.0f * (s3 * s3 - s3)) - potshift;
        vir += acc * r2;
    }
    return acc;
}

__device__ __forceinline__ uint2 ld_stream_uint2(const uint2 *p)
{
    uint2 r;
    asm("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(r.x), "=r"(r.y) : "l"(p));
    return r;
}

template <int T, bool REC, int MODE, int PREC>
__global__ void __launch_bounds__(FT_THREADS, REC ? 2 : 4) k_force_tile(FmDev d)
{
    constexpr bool NEEDW = (PREC & 6) != 0;  // Mie types / Soddemann bead flags ride in w
    constexpr bool LJ32 = PREC == 1;         // plain LJ, FP32 pair magnitude
    constexpr int R = NEEDW ? 4 : 3;
    constexpr int G = 32 / T;                // owners per warp per pass
    extern __shared__ double stg[];
    __shared__ int s_off[TILE_NSEGP];
    __shared__ int s_start[TILE_NSEG];
    __shared__ int s_code[TILE_NSEG];
    __shared__ int s_opre[9], s_ostart[8];
    __shared__ int s_blk, s_frozen, s_onext;
    pdl_enter();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_frozen = frozen(d) ? 1 : 0;
    // the dummy candidate after the capacity: far from every owner (the
    // staging below never writes index ucap)
    if (tid < R) stg[tile_woff(d.tile_ucap, R) + 32 * tid] = tid < 3 ? 1e30 : 1.0;
    __syncthreads();
    if (s_frozen) return;
    const int pset = d.sc->pset;
    const double4 *__restrict__ P = cur_pos(d, pset);
    const int sub = lane % T, og = lane / T;
    const unsigned dummy = (unsigned)tile_boff(d.tile_ucap, R);
    const unsigned lim2 = dummy | (dummy << 16);  // no byte offset beyond the dummy's
    const char *sbase = reinterpret_cast<const char *>(stg);
    const double Lx = d.L[0], Ly = d.L[1], Lz = d.L[2];
    const double rc2 = d.rc2;
    double m2max = 0.0;
    for (;;) {
        if (tid == 0) {
            const int b = atomicAdd(&d.sc->tile_next, 1);
            // every CTA takes exactly one number past the last block; the CTA
            // that takes the very last one resets the counter for the next launch
            if (b == d.tile_nblk + (int)gridDim.x - 1) d.sc->tile_next = 0;
            s_blk = b;
            s_onext = 0;
        }
        __syncthreads();
        const int blk = s_blk;
        if (blk >= d.tile_nblk) break;
        const int bx = blk % d.tile_nb[0], by = (blk / d.tile_nb[0]) % d.tile_nb[1];
        const int bz = blk / (d.tile_nb[0] * d.tile_nb[1]);
        const int x0 = 2 * bx, y0 = 2 * by, z0 = 2 * bz;
        if (tid < TILE_NSEG) {
            int st, cnt, code;
            tile_segment(d.ne, d.cell_start, x0, y0, z0, tid, st, cnt, code);
            s_start[tid] = st;
            s_code[tid] = code;
        }
        if (tid < TILE_NSEGP) s_off[tid] = d.blk_off[(size_t)blk * TILE_NSEGP + tid];
        if (warp == FT_WARPS - 1) {  // the block's owner cells a + 2b + 4c and their prefix
            int cnt = 0, st = 0;
            if (lane < 8) {
                const int x = x0 + (lane & 1), yy = y0 + ((lane >> 1) & 1), z = z0 + (lane >> 2);
                if (x < d.ne[0] && yy < d.ne[1] && z < d.ne[2]) {
                    const int c = x + d.ne[0] * (yy + d.ne[1] * z);
                    st = d.cell_start[c];
                    cnt = d.cell_start[c + 1] - st;
                }
            }
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (lane < 8) { s_opre[lane + 1] = incl; s_ostart[lane] = st; }
            if (lane == 0) s_opre[0] = 0;
        }
        __syncthreads();
        // stage, two candidates per thread per pass (both loads in flight); a
        // block above the capacity was refused by k_blk_seg before the build
        const int U = min(s_off[TILE_NSEG], d.tile_ucap);
        for (int c0 = tid; c0 < U; c0 += 2 * FT_THREADS) {
            double4 p[2];
            int code[2], cc[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int c = min(c0 + h * FT_THREADS, U - 1);  // a repeat of the last is harmless
                int k = 0;  // segment containing c: largest k with s_off[k] <= c
#pragma unroll
                for (int step = 64; step > 0; step >>= 1)
                    if (k + step < TILE_NSEG && s_off[k + step] <= c) k += step;
                p[h] = ldg_pos(P + s_start[k] + (c - s_off[k]));
                code[h] = s_code[k];
                cc[h] = c;
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int w = tile_woff(cc[h], R);
                stg[w] = image(p[h].x, (code[h] & 3) - 1, Lx);
                stg[w + 32] = image(p[h].y, ((code[h] >> 2) & 3) - 1, Ly);
                stg[w + 64] = image(p[h].z, ((code[h] >> 4) & 3) - 1, Lz);
                if (NEEDW) stg[w + 96] = p[h].w;
            }
        }
        __syncthreads();
        const int nown = s_opre[8];
        double pacc[RS_N];
#pragma unroll
        for (int q = 0; q < RS_N; q++) pacc[q] = 0.0;
        // owner groups: handed out from a shared counter (the warps of a block
        // finish together), or in a fixed order on record steps so that the
        // block's record partial is summed in the same order every time
        for (int pass = 0;; pass++) {
            int base;
            if (REC) {
                base = (warp + pass * FT_WARPS) * G;
            } else {
                if (lane == 0) base = atomicAdd(&s_onext, G);
                base = __shfl_sync(0xffffffffu, base, 0);
            }
            if (base >= nown) break;
            const int k = base + og;
            const bool act = k < nown;
            int i = 0;
            if (act) {
                int oc = 0;
#pragma unroll
                for (int q = 1; q < 8; q++) oc += k >= s_opre[q] ? 1 : 0;
                i = s_ostart[oc] + (k - s_opre[oc]);
            }
            double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0, vir = 0.0;
            double rf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            double4 pi = make_double4(0.0, 0.0, 0.0, 0.0);
            if (act) {
                pi = ldg_pos(P + i);
                const int nch = (d.nnbr[i] + 4 * T - 1) / (4 * T);  // rows are padded to whole chunks
                const uint2 *row = reinterpret_cast<const uint2 *>(d.nbr16 + tile_row16(i, d.maxn16)) + sub;
                for (int c = 0; c < nch; c++) {
                    uint2 e = ld_stream_uint2(row + c * T);
                    e.x = __vminu2(e.x, lim2);
                    e.y = __vminu2(e.y, lim2);
                    const unsigned off[4] = {e.x & 0xffffu, e.x >> 16, e.y & 0xffffu, e.y >> 16};
                    double xj[4], yj[4], zj[4], wj[4];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const double *pj = reinterpret_cast<const double *>(sbase + off[q]);
                        xj[q] = pj[0];
                        yj[q] = pj[32];
                        zj[q] = pj[64];
                        wj[q] = NEEDW ? pj[96] : 0.0;
                    }
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const double dx = __dsub_rn(pi.x, xj[q]);
                        const double dy = __dsub_rn(pi.y, yj[q]);
                        const double dz = __dsub_rn(pi.z, zj[q]);
                        const double r2 = norm2_rn(dx, dy, dz);
                        if (r2 < rc2) {
                            double acc;
                            if (LJ32) acc = lj32_pair<REC>(r2, dx, dy, dz, d.potshift, fx, fy, fz, pe, vir);
                            else acc = pair_acc<PREC, REC>(d, r2, dx, dy, dz, pi.w, wj[q], fx, fy, fz, pe, vir);
                            if (REC && d.pressure) add_rf(rf, acc, dx, dy, dz);
                        }
                    }
                }
            }
            if (T > 1) {
#pragma unroll
                for (int o = T / 2; o > 0; o >>= 1) {
                    fx += __shfl_xor_sync(0xffffffffu, fx, o);
                    fy += __shfl_xor_sync(0xffffffffu, fy, o);
                    fz += __shfl_xor_sync(0xffffffffu, fz, o);
                    if (REC) {
                        pe += __shfl_xor_sync(0xffffffffu, pe, o);
                        vir += __shfl_xor_sync(0xffffffffu, vir, o);
                        if (d.pressure) {
#pragma unroll
                            for (int q = 0; q < 6; q++) rf[q] += __shfl_xor_sync(0xffffffffu, rf[q], o);
                        }
                    }
                }
            }
            if (act && sub == 0) {
                double part[RS_N];
#pragma unroll
                for (int q = 0; q < RS_N; q++) part[q] = 0.0;
                const double m2 = owner_finish<REC, MODE, PREC>(d, pset, P, i, fx, fy, fz, pe, vir, part, rf);
                m2max = fmax(m2max, m2);
                if (REC) {
#pragma unroll
                    for (int q = 0; q < RS_N; q++)
                        pacc[q] = q == RS_PEMAX ? fmax(pacc[q], part[q]) : pacc[q] + part[q];
                }
            }
        }
        if (REC) block_partials(d, pacc, blk);
        __syncthreads();  // the next block overwrites the staging
    }
    if (MODE >= 2) block_vmax2(d, m2max);
}

// Decodes tiled rows into the generic int32 layout (rows of maxn at out),
// owner by owner: its block from its cell (cell_start), each offset back to
// a staging position, its segment by the block's prefix, and the segment's
// slot and image code (test hooks only).
__global__ void k_tile_to_generic(FmDev d, int32_t *out, int maxn)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    int lo = 0, hi = d.ncell - 1;  // largest c with cell_start[c] <= i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (d.cell_start[mid] <= i) lo = mid; else hi = mid - 1;
    }
    const int c = lo;
    const int cx = c % d.ne[0], cy = (c / d.ne[0]) % d.ne[1], cz = c / (d.ne[0] * d.ne[1]);
    const int blk = tile_block_of(d.tile_nb, cx, cy, cz);
    const int32_t *off = d.blk_off + (size_t)blk * TILE_NSEGP;
    const int cnt = min(d.nnbr[i], maxn);
    const uint16_t *row = d.nbr16 + tile_row16(i, d.maxn16);
    for (int k = 0; k < cnt; k++) {
        const int cand = tile_cand(row[tile_pos16(k, d.tile_T)], d.tile_R);
        int s = 0;
        for (int step = 64; step > 0; step >>= 1)
            if (s + step < TILE_NSEG && off[s + step] <= cand) s += step;
        int st, n, code;
        tile_segment(d.ne, d.cell_start, cx & ~1, cy & ~1, cz & ~1, s, st, n, code);
        out[nb_row(i, maxn) + nb_col(k)] = (st + (cand - off[s])) | (code << NB_SHIFT_BITS);
    }
}

// Neumaier-compensated reduction of the per-block partials into one record
// (evaluate_macroscopic_properties, simulation_record.f90:1205-1314).
constexpr int REC_THREADS = 256;
__global__ void __launch_bounds__(REC_THREADS) k_record(FmDev d, int iter, double simtime)
{
    pdl_enter();
    if (frozen(d)) return;
    __shared__ double ssum[RS_N][REC_THREADS], scmp[RS_N][REC_THREADS];
    double sum[RS_N], cmp[RS_N];
    for (int k = 0; k < RS_N; k++) { sum[k] = 0.0; cmp[k] = 0.0; }
    for (int b = threadIdx.x; b < d.nblocks_force; b += REC_THREADS) {
        for (int k = 0; k < RS_N; k++) {
            double x = d.partial[(size_t)b * RS_N + k];
            if (k == RS_PEMAX) { sum[k] = fmax(sum[k], x); continue; }
            double t = sum[k] + x;
            cmp[k] += fabs(sum[k]) >= fabs(x) ? (sum[k] - t) + x : (x - t) + sum[k];
            sum[k] = t;
        }
    }
    for (int k = 0; k < RS_N; k++) { ssum[k][threadIdx.x] = sum[k]; scmp[k][threadIdx.x] = cmp[k]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[RS_N];
        for (int k = 0; k < RS_N; k++) {
            double s = 0.0, c = 0.0;
            if (k == RS_PEMAX) {
                for (int q = 0; q < REC_THREADS; q++) s = fmax(s, ssum[k][q]);
                tot[k] = s;
                continue;
            }
            for (int q = 0; q < REC_THREADS; q++) {
                double x = ssum[k][q];
                double t = s + x;
                c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
                s = t;
                c += scmp[k][q];
            }
            tot[k] = s + c;
        }
        const double gnp = (double)d.n;
        FmRecord r;
        r.iter = iter;
        r.pad_ = 0;
        r.simtime = simtime;
        r.vsum = tot[RS_VSUM];
        r.mv2sum = tot[RS_MV2];
        r.virial = tot[RS_VIR];
        r.kinenergy = (0.5 * r.mv2sum) / gnp;
        r.potenergy = (0.5 * tot[RS_PE]) / gnp + d.pot_slrc;
        r.totenergy = r.kinenergy + r.potenergy;
        r.temperature = r.mv2sum / (3.0 * gnp);
        r.pressure = (d.density / (gnp * 3.0)) * (r.mv2sum + r.virial / 2.0) + d.p_slrc;
        int slot = d.sc->nrec_pending % d.rec_cap;
        d.rec[slot] = r;
        d.sc->nrec_pending += 1;
        if (d.pressure) {  // Pxy = Pxy + Pxytemp / volume (simulation_record.f90:3213-3217)
            const double volume = d.L[0] * d.L[1] * d.L[2];
            for (int q = 0; q < 6; q++) d.sc->pacc[q] += tot[RS_PXX + q] / volume;
            d.sc->pcount += 1;
        }
        if (tot[RS_PEMAX] > 10000.0) raise_status(d, ST_PE, iter);
    }
}

// Record partials from per-molecule arrays and current velocities
// (evaluate_macroscopic_properties reads potenergymol, virialmol and v).
constexpr int MACRO_THREADS = 256;
__global__ void __launch_bounds__(MACRO_THREADS) k_macro_partials(FmDev d)
{
    pdl_enter();
    if (frozen(d)) return;
    int i = blockIdx.x * MACRO_THREADS + threadIdx.x;
    double part[RS_N] = {};
    if (i < d.n) {
        double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
        if (d.integrator == 0) {  // leap-frog records v + a dt/2
            vx = __dadd_rn(vx, __dmul_rn(__dmul_rn(0.5, d.ax[i]), d.dt));
            vy = __dadd_rn(vy, __dmul_rn(__dmul_rn(0.5, d.ay[i]), d.dt));
            vz = __dadd_rn(vz, __dmul_rn(__dmul_rn(0.5, d.az[i]), d.dt));
        }
        const double mass = d.mie ? d.mie_mass[mie_type(cur_pos(d, d.sc->pset)[i].w) - 1] : 1.0;
        part[RS_PE] = d.pe[i];
        part[RS_VIR] = d.vir[i];
        part[RS_MV2] = mass * norm2_rn(vx, vy, vz);
        part[RS_VSUM] = mass * __dadd_rn(__dadd_rn(vx, vy), vz);
        part[RS_PEMAX] = d.pe[i];
        if (d.pressure) {
            const double *q = d.rf6 + 6 * (size_t)i;
            const double rf[6] = {q[0], q[1], q[2], q[3], q[4], q[5]};
            pressure_part(part, vx, vy, vz, rf);
        }
    }
    block_partials<MACRO_THREADS>(d, part, blockIdx.x);
}

// ---------------------------------------------------------------------------
// all pairs with per-axis minimum image (simulation_compute_forces_LJ_AP,
// simulation_compute_forces.f90:280-341), both sides evaluated per molecule
// ---------------------------------------------------------------------------

constexpr int AP_THREADS = 128;
template <bool REC, int MODE, int PREC>
__global__ void __launch_bounds__(AP_THREADS) k_all_pairs(FmDev d)
{
    pdl_enter();
    if (frozen(d)) return;
    const int pset = d.sc->pset;
    const double4 *P = cur_pos(d, pset);
    const int i = blockIdx.x * AP_THREADS + threadIdx.x;
    const bool active = i < d.n;
    __shared__ double4 tile[AP_THREADS];
    double4 pi = active ? P[i] : make_double4(0, 0, 0, 0);
    double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0, vir = 0.0;
    for (int t0 = 0; t0 < d.n; t0 += AP_THREADS) {
        int j0 = t0 + threadIdx.x;
        if (j0 < d.n) tile[threadIdx.x] = P[j0];
        __syncthreads();
        int m = min(AP_THREADS, d.n - t0);
        if (active) {
            for (int q = 0; q < m; q++) {
                if (t0 + q == i) continue;
                double4 pj = tile[q];
                double r[3] = {__dsub_rn(pi.x, pj.x), __dsub_rn(pi.y, pj.y), __dsub_rn(pi.z, pj.z)};
                double r2 = 0.0;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    if (fabs(r[k]) > d.hd[k]) r[k] = __dsub_rn(r[k], copysign(d.L[k], r[k]));
                    r2 = __dadd_rn(r2, __dmul_rn(r[k], r[k]));
                }
                if (r2 < d.rc2) pair_acc<PREC, REC>(d, r2, r[0], r[1], r[2], pi.w, pj.w, fx, fy, fz, pe, vir);
            }
        }
        __syncthreads();
    }
    double part[RS_N] = {};
    double m2 = 0.0;
    const double rf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // simulation_compute_forces_LJ_AP records no rf
    if (active) m2 = epilogue<REC, MODE, (PREC & 2) != 0>(d, pset, i, pi, fx, fy, fz, pe, vir, part, rf);
    if (REC) block_partials<AP_THREADS>(d, part, blockIdx.x);
    if (MODE >= 2) block_vmax2(d, m2);
}

// ---------------------------------------------------------------------------
// test hooks and layout conversion
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27; x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

__global__ void k_pair_digest(FmDev d, const int32_t *glob_of_upload)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t h = 0ull;
    long long cnt = 0;
    if (i < d.n) {
        int gi = glob_of_upload[d.slot_of[i]];
        const int32_t *L = d.nbr + nb_row(i, d.maxn);
        for (int k = 0; k < d.nnbr[i]; k++) {
            int e = L[nb_col(k)];
            int j = e & NB_INDEX_MASK;
            int code6 = e >> NB_SHIFT_BITS;
            int sx = (code6 & 3) - 1, sy = ((code6 >> 2) & 3) - 1, sz = ((code6 >> 4) & 3) - 1;
            int code = (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
            int gj = glob_of_upload[d.slot_of[j]];
            if (code == 13) {
                if (gi < gj) {  // both directions are stored; count the unordered pair once
                    h += mix64(((uint64_t)(uint32_t)gi << 32) ^ (uint64_t)(uint32_t)gj);
                    cnt++;
                }
            } else {
                h += mix64((((uint64_t)(uint32_t)gi << 32) ^ (uint64_t)(uint32_t)gj) * 31ull + (uint64_t)code + 0x9e3779b97f4a7c15ull);
                cnt++;
            }
        }
    }
    h = warp_sum<unsigned long long>(h);
    cnt = warp_sum<long long>(cnt);
    if ((threadIdx.x & 31) == 0 && (h || cnt)) {
        atomicAdd((unsigned long long *)&d.sc->digest, (unsigned long long)h);
        atomicAdd((unsigned long long *)&d.sc->digest_n, (unsigned long long)cnt);
    }
}

// Types of an uploaded state (slots still equal upload indices).
// w of each position from the Mie type (moltype) and the Soddemann bead flag
// (solvent_flag 1: 1 for a chain bead, 0 for a solvent molecule, chainID 0):
// the type, the flag, or the type + 32 x the flag with both.  Run after either
// is uploaded, while slots still equal upload indices; a part not uploaded
// yet reads as 0 (type) or the zeroed chain ids.
__global__ void k_set_w(FmDev d)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= d.n) return;
    const int type = d.mie && d.mie_type_up ? d.mie_type_up[u] : 0;
    const int flag = d.solvent ? (d.chain[u] != 0 ? 1 : 0) : 0;
    cur_pos(d, d.sc->pset)[u].w = (double)(type + (d.mie ? 32 : 1) * flag);
}

// upload order u -> slot u (uploads start in upload order)
__global__ void k_scatter_state(FmDev d, const double *r3, const double *v3, const double *a3)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= d.n) return;
    double4 *P = cur_pos(d, d.sc->pset);
    P[u] = make_double4(r3[3 * (size_t)u], r3[3 * (size_t)u + 1], r3[3 * (size_t)u + 2],
                        d.mie ? (double)d.mie_type_up[u] : 0.0);
    d.vx[u] = v3[3 * (size_t)u]; d.vy[u] = v3[3 * (size_t)u + 1]; d.vz[u] = v3[3 * (size_t)u + 2];
    if (a3) { d.ax[u] = a3[3 * (size_t)u]; d.ay[u] = a3[3 * (size_t)u + 1]; d.az[u] = a3[3 * (size_t)u + 2]; }
    else { d.ax[u] = 0.0; d.ay[u] = 0.0; d.az[u] = 0.0; }
    d.slot_of[u] = u;
}

__global__ void k_gather_state(FmDev d, double *r3, double *v3, double *a3, int32_t *uidx_out, double *pe,
                               double *vir)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n) return;
    int u = d.slot_of[s];
    const double4 *P = cur_pos(d, d.sc->pset);
    if (r3) { double4 p = P[s]; r3[3 * (size_t)u] = p.x; r3[3 * (size_t)u + 1] = p.y; r3[3 * (size_t)u + 2] = p.z; }
    if (v3) { v3[3 * (size_t)u] = d.vx[s]; v3[3 * (size_t)u + 1] = d.vy[s]; v3[3 * (size_t)u + 2] = d.vz[s]; }
    if (a3) { a3[3 * (size_t)u] = d.ax[s]; a3[3 * (size_t)u + 1] = d.ay[s]; a3[3 * (size_t)u + 2] = d.az[s]; }
    if (uidx_out) uidx_out[s] = u;
    if (pe) pe[u] = d.pe[s];
    if (vir) vir[u] = d.vir[s];
}

inline int nblk(int n, int t) { return (n + t - 1) / t; }

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------


void launch_reset_scalars(const FmDev &d, cudaStream_t st) { k_reset_scalars<<<1, 1, 0, st>>>(d); }
void launch_move1(const FmDev &d, cudaStream_t st) { pdl_launch(k_move1, nblk(d.n, 256), 256, st, d); }
void launch_move2(const FmDev &d, cudaStream_t st) { pdl_launch(k_move2, nblk(d.n, 256), 256, st, d); }
void launch_vmax(const FmDev &d, cudaStream_t st) { pdl_launch(k_vmax, nblk(d.n, 256), 256, st, d); }
void launch_move_lfv(const FmDev &d, cudaStream_t st) { pdl_launch(k_move_lfv, nblk(d.n, 256), 256, st, d); }
void launch_disp(const FmDev &d, cudaStream_t st) { pdl_launch(k_disp, nblk(d.n, 256), 256, st, d); }

void launch_decide_graph(const FmDev &d, int flip, int crit, int fixed_rebuild, double half_min_delta,
                         cudaGraphConditionalHandle cond, int body_kernels, cudaStream_t st)
{
    k_decide_graph<<<1, 1, 0, st>>>(d, flip, crit, fixed_rebuild > 0 ? fixed_rebuild : 1, half_min_delta, cond,
                                    body_kernels);
}

void launch_set_graph_iter(const FmDev &d, int iter, cudaStream_t st) { k_set_graph_iter<<<1, 1, 0, st>>>(d, iter); }

void launch_decide(const FmDev &d, int iter, int flip, int crit, int fixed_rebuild, double half_min_delta,
                   cudaStream_t st)
{
    pdl_launch(k_decide, 1, 1, st, d, iter, flip, crit, fixed_rebuild > 0 ? fixed_rebuild : 1, half_min_delta);
}
// Gated kernels run grid-stride loops on a bounded grid, so that a launch the
// device decision turns into a no-op costs a few microseconds at most.
constexpr int kSMs = 148;
inline int sgrid(int n, int t, int per_sm) { return std::min(nblk(n, t), kSMs * per_sm); }

void launch_wrap_bin(const FmDev &d, int wrap, int bin, int gated, int iter, cudaStream_t st)
{
    pdl_launch(k_wrap_bin, sgrid(d.n, 256, 8), 256, st, d, wrap, bin, gated, iter);
}
int scan_tiles(int ncell) { return nblk(ncell, SCAN_TILE); }
void launch_scan_cells(const FmDev &d, int gated, cudaStream_t st)
{
    pdl_launch(k_scan_tiles, scan_tiles(d.ncell), SCAN_THREADS, st, d, gated);
    pdl_launch(k_scan_apply, scan_tiles(d.ncell), SCAN_THREADS, st, d, gated);
}
void launch_scatter(const FmDev &d, int gated, cudaStream_t st)
{
    pdl_launch(k_scatter, sgrid(d.n, 256, 8), 256, st, d, gated);
    pdl_launch(k_sort_cells, sgrid(d.ncell, SORT_WARPS, 8), 32 * SORT_WARPS, st, d, gated);
}
void launch_reorder(const FmDev &d, int gated, double4 *tpos, int32_t *tuidx, cudaStream_t st)
{
    pdl_launch(k_reorder_gather, sgrid(d.n, 256, 8), 256, st, d, gated, tpos, tuidx);
    pdl_launch(k_reorder_copy, sgrid(d.n, 256, 8), 256, st, d, gated, tpos, tuidx);
}
// The list build walks the cells grid-stride with every block resident (one
// wave: a second partial wave would double the kernel's time).
template <bool POLY, bool BLOCKS, bool TILE>
static size_t build_smem_bytes()
{
    using Shared = typename std::conditional<BLOCKS, BlockShared<POLY, TILE>, BuildShared<POLY, TILE>>::type;
    return sizeof(Shared) * NB_WARPS;
}

template <bool POLY, bool BLOCKS, bool TILE>
static int build_grid(int nwork)
{
    static int resident = 0;
    if (resident == 0) {
        int dev = 0, nsm = kSMs, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_build_nlist<POLY, BLOCKS, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)build_smem_bytes<POLY, BLOCKS, TILE>());
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build_nlist<POLY, BLOCKS, TILE>, NB_THREADS,
                                                      build_smem_bytes<POLY, BLOCKS, TILE>());
        resident = std::max(nsm, 1) * std::max(per_sm, 1);
    }
    return std::min(nblk(nwork, NB_WARPS), resident);
}

template <bool POLY, bool BLOCKS, bool TILE>
static void launch_build_t(const FmDev &d, int nwork, int gated, int iter, cudaStream_t st)
{
    const int g = build_grid<POLY, BLOCKS, TILE>(nwork);  // (sets the kernel's shared-memory attribute once)
    pdl_launch_smem(k_build_nlist<POLY, BLOCKS, TILE>, g, NB_THREADS, build_smem_bytes<POLY, BLOCKS, TILE>(), st, d,
                    gated, iter);
}

void launch_build_nlist(const FmDev &d, int gated, int iter, cudaStream_t st)
{
    cudaMemsetAsync(&d.sc->build_next, 0, sizeof(int32_t), st);
    const int nb = ((d.ne[0] + 1) / 2) * ((d.ne[1] + 1) / 2) * ((d.ne[2] + 1) / 2);
    const int nw = d.build_blocks ? nb : d.ncell;
    switch ((d.potential_flag == 1 ? 4 : 0) + (d.build_blocks ? 2 : 0) + (d.tile ? 1 : 0)) {
    case 0: launch_build_t<false, false, false>(d, nw, gated, iter, st); break;
    case 1: launch_build_t<false, false, true>(d, nw, gated, iter, st); break;
    case 2: launch_build_t<false, true, false>(d, nw, gated, iter, st); break;
    case 3: launch_build_t<false, true, true>(d, nw, gated, iter, st); break;
    case 4: launch_build_t<true, false, false>(d, nw, gated, iter, st); break;
    case 5: launch_build_t<true, false, true>(d, nw, gated, iter, st); break;
    case 6: launch_build_t<true, true, false>(d, nw, gated, iter, st); break;
    default: launch_build_t<true, true, true>(d, nw, gated, iter, st); break;
    }
}

void launch_angular_order(const FmDev &d, int gated, int iter, cudaStream_t st)
{
    pdl_launch(k_angular_order, sgrid(d.n, 256, 8), 256, st, d, gated, iter);
}

void launch_set_funcy(const FmDev &d, const int32_t *funcy_up, cudaStream_t st)
{
    k_set_funcy<<<nblk(d.n, 256), 256, 0, st>>>(d, funcy_up);
}

void launch_blk_seg(const FmDev &d, int gated, int iter, cudaStream_t st)
{
    pdl_launch(k_blk_seg, sgrid(d.tile_nblk, BS_THREADS / 32, 8), BS_THREADS, st, d, gated, iter);
}

// Staging capacity of the tiled force kernel: list entries are 16-bit byte
// offsets into the staging, so it holds at most tile_ucap_max(R) candidates
// (2720 for x y z, 2016 with w) plus the dummy -- at most ~64 KB.
constexpr int TILE_SMEM_MAX = 232448 - 4096;
int tile_ucap_limit(int R) { return tile_ucap_max(R); }
size_t tile_smem_bytes(const FmDev &d) { return (size_t)tile_stage_doubles(d.tile_ucap, d.tile_R) * 8; }

template <int T, bool REC, int MODE, int PREC>
static void launch_force_tile_k(const FmDev &d, cudaStream_t st)
{
    auto k = k_force_tile<T, REC, MODE, PREC>;
    static size_t smem_set = 0;
    static int grid_for = -1, grid = 0;
    const size_t smem = tile_smem_bytes(d);
    if (smem_set == 0) {
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, TILE_SMEM_MAX);
        smem_set = 1;
    }
    if (grid_for != (int)smem) {  // resident CTAs at this staging size
        int dev = 0, nsm = kSMs, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, FT_THREADS, smem);
        grid = std::max(nsm, 1) * std::max(per_sm, 1);
        grid_for = (int)smem;
    }
    pdl_launch_smem(k, std::min(grid, d.tile_nblk), FT_THREADS, smem, st, d);
}

template <int T>
static void launch_force_tile(const FmDev &d, int record, int mode, cudaStream_t st)
{
#define FM_TILE_CASE(R, M)                                                          \
    if (record == R && mode == M) {                                                 \
        switch (d.precision + 2 * d.mie + 4 * d.solvent) {                          \
        case 0: launch_force_tile_k<T, R, M, 0>(d, st); break;                      \
        case 1: launch_force_tile_k<T, R, M, 1>(d, st); break;                      \
        case 2: launch_force_tile_k<T, R, M, 2>(d, st); break;                      \
        case 3: launch_force_tile_k<T, R, M, 3>(d, st); break;                      \
        case 4: launch_force_tile_k<T, R, M, 4>(d, st); break;                      \
        case 5: launch_force_tile_k<T, R, M, 5>(d, st); break;                      \
        case 6: launch_force_tile_k<T, R, M, 6>(d, st); break;                      \
        default: launch_force_tile_k<T, R, M, 7>(d, st); break;                     \
        }                                                                           \
        return;                                                                     \
    }
    FM_TILE_CASE(0, 0) FM_TILE_CASE(0, 1) FM_TILE_CASE(0, 2) FM_TILE_CASE(0, 3)
    FM_TILE_CASE(1, 0) FM_TILE_CASE(1, 1) FM_TILE_CASE(1, 2) FM_TILE_CASE(1, 3)
#undef FM_TILE_CASE
}

void launch_tile_to_generic(const FmDev &d, int32_t *out, int maxn, cudaStream_t st)
{
    k_tile_to_generic<<<nblk(d.n, 128), 128, 0, st>>>(d, out, maxn);
}

int force_blocks(int n, int tpm) { return nblk(n * tpm, FORCE_THREADS); }
int all_pairs_blocks(int n) { return nblk(n, AP_THREADS); }

template <int TPM>
static void launch_force_tpm(const FmDev &d, int record, int mode, cudaStream_t st)
{
    const int g = force_blocks(d.n, TPM);
#define FM_FORCE_CASE(R, M)                                                                     \
    if (record == R && mode == M) {                                                             \
        switch (d.precision + 2 * d.mie + 4 * d.solvent) {                                      \
        case 0: pdl_launch(k_force<TPM, R, M, 0>, g, FORCE_THREADS, st, d); break;                   \
        case 1: pdl_launch(k_force<TPM, R, M, 1>, g, FORCE_THREADS, st, d); break;                   \
        case 2: pdl_launch(k_force<TPM, R, M, 2>, g, FORCE_THREADS, st, d); break;                   \
        case 3: pdl_launch(k_force<TPM, R, M, 3>, g, FORCE_THREADS, st, d); break;                   \
        case 4: pdl_launch(k_force<TPM, R, M, 4>, g, FORCE_THREADS, st, d); break;                   \
        case 5: pdl_launch(k_force<TPM, R, M, 5>, g, FORCE_THREADS, st, d); break;                   \
        case 6: pdl_launch(k_force<TPM, R, M, 6>, g, FORCE_THREADS, st, d); break;                   \
        default: pdl_launch(k_force<TPM, R, M, 7>, g, FORCE_THREADS, st, d); break;                  \
        }                                                                                       \
        return;                                                                                 \
    }
    FM_FORCE_CASE(0, 0) FM_FORCE_CASE(0, 1) FM_FORCE_CASE(0, 2) FM_FORCE_CASE(0, 3)
    FM_FORCE_CASE(1, 0) FM_FORCE_CASE(1, 1) FM_FORCE_CASE(1, 2) FM_FORCE_CASE(1, 3)
#undef FM_FORCE_CASE
}

void launch_force(const FmDev &d, int record, int mode, int tpm, cudaStream_t st)
{
    if (d.tile) {
        if (d.tile_T == 4) launch_force_tile<4>(d, record, mode, st);
        else launch_force_tile<8>(d, record, mode, st);
        return;
    }
    switch (tpm) {
    case 1: launch_force_tpm<1>(d, record, mode, st); break;
    case 2: launch_force_tpm<2>(d, record, mode, st); break;
    case 4: launch_force_tpm<4>(d, record, mode, st); break;
    case 16: launch_force_tpm<16>(d, record, mode, st); break;
    default: launch_force_tpm<8>(d, record, mode, st); break;
    }
}

void launch_all_pairs(const FmDev &d, int record, int mode, cudaStream_t st)
{
    const int g = all_pairs_blocks(d.n);
#define FM_AP_CASE(R, M)                                                            \
    if (record == R && mode == M) {                                                 \
        switch (d.precision + 2 * d.mie) {                                          \
        case 0: pdl_launch(k_all_pairs<R, M, 0>, g, AP_THREADS, st, d); break;           \
        case 1: pdl_launch(k_all_pairs<R, M, 1>, g, AP_THREADS, st, d); break;           \
        case 2: pdl_launch(k_all_pairs<R, M, 2>, g, AP_THREADS, st, d); break;           \
        default: pdl_launch(k_all_pairs<R, M, 3>, g, AP_THREADS, st, d); break;          \
        }                                                                           \
        return;                                                                     \
    }
    FM_AP_CASE(0, 0) FM_AP_CASE(0, 1) FM_AP_CASE(0, 2) FM_AP_CASE(0, 3)
    FM_AP_CASE(1, 0) FM_AP_CASE(1, 1) FM_AP_CASE(1, 2) FM_AP_CASE(1, 3)
#undef FM_AP_CASE
}

int macro_blocks(int n) { return nblk(n, MACRO_THREADS); }
void launch_macro_partials(const FmDev &d, cudaStream_t st)
{
    pdl_launch(k_macro_partials, macro_blocks(d.n), MACRO_THREADS, st, d);
}

void launch_record(const FmDev &d, int iter, double simtime, cudaStream_t st)
{
    pdl_launch(k_record, 1, REC_THREADS, st, d, iter, simtime);
}

void launch_pair_digest(const FmDev &d, const int32_t *glob_of_upload, cudaStream_t st)
{
    k_pair_digest<<<nblk(d.n, 256), 256, 0, st>>>(d, glob_of_upload);
}

void launch_set_types(const FmDev &d, cudaStream_t st) { k_set_w<<<nblk(d.n, 256), 256, 0, st>>>(d); }

void launch_set_bead_flags(const FmDev &d, cudaStream_t st) { k_set_w<<<nblk(d.n, 256), 256, 0, st>>>(d); }

void launch_scatter_state(const FmDev &d, const double *r3, const double *v3, const double *a3, cudaStream_t st)
{
    k_scatter_state<<<nblk(d.n, 256), 256, 0, st>>>(d, r3, v3, a3);
}

void launch_gather_state(const FmDev &d, double *r3, double *v3, double *a3, int32_t *uidx, double *pe,
                         double *vir, cudaStream_t st)
{
    k_gather_state<<<nblk(d.n, 256), 256, 0, st>>>(d, r3, v3, a3, uidx, pe, vir);
}

}  // namespace fm
