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

#include "fm_common.cuh"

namespace fm {

namespace {

__device__ __forceinline__ bool frozen(const FmDev &d) { return (d.sc->status & ST_FATAL) != 0u; }

__device__ __forceinline__ void raise_status(const FmDev &d, uint32_t bit, int iter)
{
    uint32_t old = atomicOr(&d.sc->status, bit);
    if ((old & ST_FATAL) == 0u) d.sc->fail_iter = iter;
}

// |v|^2 in the reference's dot_product order, no contraction.
__device__ __forceinline__ double norm2_rn(double x, double y, double z)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// Read-only gather of x, y, z of a double4 (one 32-byte sector).
__device__ __forceinline__ double4 ldg_pos(const double4 *p)
{
    const double2 xy = __ldg(reinterpret_cast<const double2 *>(p));
    const double z = __ldg(reinterpret_cast<const double *>(p) + 2);
    return make_double4(xy.x, xy.y, z, 0.0);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
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
}

// r = (r + dt v) + (0.5 dt^2) a ; v = v + (0.5 dt) a   -- pass 1, in place.
__global__ void k_move1(FmDev d)
{
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
    if (frozen(d)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n) {
        d.vx[i] = __dadd_rn(d.vx[i], __dmul_rn(d.half_dt, d.ax[i]));
        d.vy[i] = __dadd_rn(d.vy[i], __dmul_rn(d.half_dt, d.ay[i]));
        d.vz[i] = __dadd_rn(d.vz[i], __dmul_rn(d.half_dt, d.az[i]));
    }
}

__global__ void k_vmax(FmDev d)
{
    if (frozen(d)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m2 = 0.0;
    if (i < d.n) m2 = norm2_rn(d.vx[i], d.vy[i], d.vz[i]);
    block_vmax2(d, m2);
}

// ---------------------------------------------------------------------------
// rebuild decision (simulation_checkrebuild.f90:34, 83-99, 101-103, 148-155)
// ---------------------------------------------------------------------------

__global__ void k_decide(FmDev d, int iter, int flip, int crit, int fixed_rebuild, double half_min_delta)
{
    FmScalars *s = d.sc;
    if (s->status & ST_FATAL) return;
    if (flip) s->pset ^= 1;
    int rebuild = ((iter + 1) % d.tplot) == 0 ? 1 : 0;
    if (crit == 0) {
        double vmax = sqrt(__longlong_as_double((long long)s->vmax2));
        s->rmax = __dadd_rn(s->rmax, __dmul_rn(vmax, d.dt));
        if (s->rmax > half_min_delta) rebuild = 1;
    } else if (crit == 1) {
        if ((iter % fixed_rebuild) == 0) rebuild = 1;
    }
    s->vmax2 = 0ull;
    if (rebuild) {
        s->rmax = 0.0;
        s->rebuilds += 1;
    }
    s->rebuild = rebuild;
}

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

// icell = ceiling((r + halfdomain)/cellsidelength) + 1 (1-based, halo = 1 and
// ncells+2); the 0-based extended index is the ceiling itself.
__device__ __forceinline__ int bin_axis(double x, double hd, double cs, int ne, bool &bad)
{
    double q = __ddiv_rn(__dadd_rn(x, hd), cs);
    if (!(q == q)) { bad = true; return 0; }
    int c = __double2int_ru(q);  // round toward +inf == ceiling for in-range values
    if (c < 0 || c > ne - 1) { bad = true; c = c < 0 ? 0 : ne - 1; }
    return c;
}

__global__ void k_wrap_bin(FmDev d, int wrap, int bin, int gated, int iter)
{
    if (!gate(d, gated)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    double4 *P = cur_pos(d, d.sc->pset);
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
    if (!bin) return;
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

// Exclusive scan of the per-cell counts in one block; the counts are zeroed
// so the scatter can reuse them as cursors.
constexpr int SCAN_THREADS = 1024;
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_cells(FmDev d, int gated)
{
    if (!gate(d, gated)) return;
    __shared__ int wsum[32];
    const int nc = d.ncell;
    const int per = (nc + SCAN_THREADS - 1) / SCAN_THREADS;
    const int b = threadIdx.x * per;
    const int e = min(b + per, nc);
    int local = 0;
    for (int c = b; c < e; c++) local += d.cell_count[c];
    // block exclusive scan of `local`
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int v = wsum[lane];
        int vi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, vi, o);
            if (lane >= o) vi += t;
        }
        wsum[lane] = vi - v;
    }
    __syncthreads();
    int run = wsum[w] + incl - local;
    for (int c = b; c < e; c++) {
        int k = d.cell_count[c];
        d.cell_start[c] = run;
        d.cell_count[c] = 0;
        run += k;
    }
    if (threadIdx.x == SCAN_THREADS - 1) d.cell_start[nc] = run;
}

__global__ void k_scatter(FmDev d, int gated)
{
    if (!gate(d, gated)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    int c = d.cell_of[i];
    int slot = d.cell_start[c] + atomicAdd(&d.cell_count[c], 1);
    d.perm[slot] = i;
}

// Atomics make the in-cell order arbitrary; sorting each cell by old slot
// makes the whole rebuild deterministic.
__global__ void k_sort_cells(FmDev d, int gated)
{
    if (!gate(d, gated)) return;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.ncell) return;
    int b = d.cell_start[c], e = d.cell_start[c + 1];
    for (int x = b + 1; x < e; x++) {
        int key = d.perm[x];
        int y = x - 1;
        while (y >= b && d.perm[y] > key) {
            d.perm[y + 1] = d.perm[y];
            y--;
        }
        d.perm[y + 1] = key;
    }
    d.cell_count[c] = 0;  // leave counts zeroed for the next histogram
}

// Gather into scratch in cell order, then copy back, so every array keeps
// its address (the step loop never needs to know whether a rebuild ran).
__global__ void k_reorder_gather(FmDev d, int gated, double4 *tpos, int32_t *tuidx)
{
    if (!gate(d, gated)) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n) return;
    int o = d.perm[s];
    const double4 *P = cur_pos(d, d.sc->pset);
    tpos[s] = P[o];
    d.tvx[s] = d.vx[o]; d.tvy[s] = d.vy[o]; d.tvz[s] = d.vz[o];
    d.tax[s] = d.ax[o]; d.tay[s] = d.ay[o]; d.taz[s] = d.az[o];
    tuidx[s] = d.slot_of[o];
}

__global__ void k_reorder_copy(FmDev d, int gated, const double4 *tpos, const int32_t *tuidx)
{
    if (!gate(d, gated)) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n) return;
    double4 *P = cur_pos(d, d.sc->pset);
    P[s] = tpos[s];
    d.vx[s] = d.tvx[s]; d.vy[s] = d.tvy[s]; d.vz[s] = d.tvz[s];
    d.ax[s] = d.tax[s]; d.ay[s] = d.tay[s]; d.az[s] = d.taz[s];
    d.slot_of[s] = tuidx[s];
}

// ---------------------------------------------------------------------------
// neighbour list from shared-memory cell tiles
// (pair set of assign_to_neighbourlist_halfint_opt, linklist.f90:660-804,
//  1118-1180, stored in both directions)
// ---------------------------------------------------------------------------

constexpr int NB_THREADS = 32;
constexpr int NB_STAGE = 192;

struct Seg {
    int start, count, code;  // code = (sx+1) | (sy+1)<<2 | (sz+1)<<4
};

__device__ __forceinline__ bool is_halo(int x, int ne) { return x == 0 || x == ne - 1; }

// One block per extended cell.  The reference visits every pair of adjacent
// cells of which at least one is interior exactly once (13 forward shifts
// from interior cells + 27 sweeps from halo cells); a halo cell holds the
// images of the opposite boundary cell (plus any real molecule that binned
// onto it).  Here each molecule of cell c collects, from the 27 cells around
// c that are not both halo with c, every candidate within rneighbr.
__global__ void __launch_bounds__(NB_THREADS) k_build_nlist(FmDev d, int gated, int iter)
{
    if (!gate(d, gated)) return;
    const int c = blockIdx.x;
    const int cstart = d.cell_start[c];
    const int ccount = d.cell_start[c + 1] - cstart;
    if (ccount == 0) return;
    const int ne0 = d.ne[0], ne1 = d.ne[1], ne2 = d.ne[2];
    const int cx = c % ne0, cy = (c / ne0) % ne1, cz = c / (ne0 * ne1);
    const bool chalo = is_halo(cx, ne0) || is_halo(cy, ne1) || is_halo(cz, ne2);
    const double4 *P = cur_pos(d, d.sc->pset);

    __shared__ Seg segs[54];
    __shared__ int nseg;
    __shared__ double sx[NB_STAGE], sy[NB_STAGE], sz[NB_STAGE];
    __shared__ int32_t se[NB_STAGE];

    if (threadIdx.x == 0) {
        int ns = 0;
        for (int q = 0; q < 27; q++) {
            int dx = q % 3 - 1, dy = (q / 3) % 3 - 1, dz = q / 9 - 1;
            int x2 = cx + dx, y2 = cy + dy, z2 = cz + dz;
            if (x2 < 0 || y2 < 0 || z2 < 0 || x2 >= ne0 || y2 >= ne1 || z2 >= ne2) continue;
            bool h2 = is_halo(x2, ne0) || is_halo(y2, ne1) || is_halo(z2, ne2);
            if (chalo && h2) continue;
            int c2 = x2 + ne0 * (y2 + ne1 * z2);
            int b2 = d.cell_start[c2], n2 = d.cell_start[c2 + 1] - b2;
            if (n2 > 0) segs[ns++] = Seg{b2, n2, 1 | (1 << 2) | (1 << 4)};
            if (h2) {
                // images in halo cell (x2,y2,z2) come from the interior cell on the
                // far side: low halo <- last interior cell shifted by -domain,
                // high halo <- first interior cell shifted by +domain
                int ssx = x2 == 0 ? -1 : (x2 == ne0 - 1 ? 1 : 0);
                int ssy = y2 == 0 ? -1 : (y2 == ne1 - 1 ? 1 : 0);
                int ssz = z2 == 0 ? -1 : (z2 == ne2 - 1 ? 1 : 0);
                int xs = x2 == 0 ? ne0 - 2 : (x2 == ne0 - 1 ? 1 : x2);
                int ys = y2 == 0 ? ne1 - 2 : (y2 == ne1 - 1 ? 1 : y2);
                int zs = z2 == 0 ? ne2 - 2 : (z2 == ne2 - 1 ? 1 : z2);
                int cs2 = xs + ne0 * (ys + ne1 * zs);
                int bs = d.cell_start[cs2], nsrc = d.cell_start[cs2 + 1] - bs;
                if (nsrc > 0) segs[ns++] = Seg{bs, nsrc, (ssx + 1) | ((ssy + 1) << 2) | ((ssz + 1) << 4)};
            }
        }
        nseg = ns;
    }
    __syncthreads();
    const int ns = nseg;
    const double Lx = d.L[0], Ly = d.L[1], Lz = d.L[2];
    const double rn2 = d.rn2;
    const int maxn = d.maxn;
    const int noshift = 1 | (1 << 2) | (1 << 4);

    for (int pass = 0; pass * NB_THREADS < ccount; pass++) {
        const int mine = pass * NB_THREADS + threadIdx.x;
        const bool own = mine < ccount;
        const int i = cstart + (own ? mine : 0);
        double4 pi = P[i];
        int cnt = 0;
        int32_t *out = d.nbr + (size_t)i * maxn;
        int fill = 0;
        for (int sgi = 0; sgi < ns; sgi++) {
            const Seg sg = segs[sgi];
            const int sxs = (sg.code & 3) - 1, sys = ((sg.code >> 2) & 3) - 1, szs = ((sg.code >> 4) & 3) - 1;
            int base = 0;
            while (base < sg.count) {
                int take = min(sg.count - base, NB_STAGE - fill);
                for (int t = threadIdx.x; t < take; t += NB_THREADS) {
                    int j = sg.start + base + t;
                    double4 pj = P[j];
                    // image coordinate: one FP64 add per shifted axis, as the halo copy
                    sx[fill + t] = sxs ? __dadd_rn(pj.x, sxs > 0 ? Lx : -Lx) : pj.x;
                    sy[fill + t] = sys ? __dadd_rn(pj.y, sys > 0 ? Ly : -Ly) : pj.y;
                    sz[fill + t] = szs ? __dadd_rn(pj.z, szs > 0 ? Lz : -Lz) : pj.z;
                    se[fill + t] = j | (sg.code << NB_SHIFT_BITS);
                }
                fill += take;
                base += take;
                if (fill == NB_STAGE) {
                    __syncthreads();
                    if (own) {
                        for (int q = 0; q < fill; q++) {
                            int e = se[q];
                            if ((e & NB_INDEX_MASK) == i && (e >> NB_SHIFT_BITS) == noshift) continue;
                            double dx = __dsub_rn(pi.x, sx[q]);
                            double dy = __dsub_rn(pi.y, sy[q]);
                            double dz = __dsub_rn(pi.z, sz[q]);
                            double r2 = norm2_rn(dx, dy, dz);
                            if (r2 < rn2) {
                                if (cnt < maxn) out[cnt] = e;
                                cnt++;
                            }
                        }
                    }
                    __syncthreads();
                    fill = 0;
                }
            }
        }
        __syncthreads();
        if (own) {
            for (int q = 0; q < fill; q++) {
                int e = se[q];
                if ((e & NB_INDEX_MASK) == i && (e >> NB_SHIFT_BITS) == noshift) continue;
                double dx = __dsub_rn(pi.x, sx[q]);
                double dy = __dsub_rn(pi.y, sy[q]);
                double dz = __dsub_rn(pi.z, sz[q]);
                double r2 = norm2_rn(dx, dy, dz);
                if (r2 < rn2) {
                    if (cnt < maxn) out[cnt] = e;
                    cnt++;
                }
            }
            d.nnbr[i] = cnt < maxn ? cnt : maxn;
            atomicMax(&d.sc->max_nbr, cnt);
            if (cnt > maxn) raise_status(d, ST_NLIST, iter);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// forces (simulation_compute_forces_LJ_neigbr*, simulation_compute_forces.f90
// :551-726) fused with move(2) and the next move(1)
// ---------------------------------------------------------------------------

constexpr int FORCE_THREADS = 256;

// Block reduction of the record partials; row blockIdx.x of d.partial.
__device__ __forceinline__ void block_partials(const FmDev &d, double v[RS_N])
{
    __shared__ double ws[RS_N][FORCE_THREADS / 32];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < RS_N; k++) {
        double x = k == RS_PEMAX ? warp_max(v[k]) : warp_sum(v[k]);
        if (l == 0) ws[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < RS_N) {
        int k = threadIdx.x;
        double acc = ws[k][0];
        for (int q = 1; q < FORCE_THREADS / 32; q++) acc = k == RS_PEMAX ? fmax(acc, ws[k][q]) : acc + ws[k][q];
        d.partial[(size_t)blockIdx.x * RS_N + k] = acc;
    }
}

template <int TPM, bool REC, int MODE, int PREC>
__global__ void __launch_bounds__(FORCE_THREADS) k_force(FmDev d)
{
    if (frozen(d)) return;
    const int pset = d.sc->pset;
    const double4 *__restrict__ P = cur_pos(d, pset);
    const int gt = blockIdx.x * FORCE_THREADS + threadIdx.x;
    const int i = gt / TPM;
    const int lane = gt % TPM;
    const bool active = i < d.n;
    double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0, vir = 0.0;
    if (active) {
        const double4 pi = P[i];
        const int cnt = d.nnbr[i];
        const int32_t *__restrict__ L = d.nbr + (size_t)i * d.maxn;
        const double Lx = d.L[0], Ly = d.L[1], Lz = d.L[2];
        const double rc2 = d.rc2;
        for (int k = lane; k < cnt; k += TPM) {
            const int e = __ldg(L + k);
            const double4 pj = ldg_pos(P + (e & NB_INDEX_MASK));
            const int code = e >> NB_SHIFT_BITS;
            const int ssx = (code & 3) - 1, ssy = ((code >> 2) & 3) - 1, ssz = ((code >> 4) & 3) - 1;
            const double xj = ssx ? __dadd_rn(pj.x, ssx > 0 ? Lx : -Lx) : pj.x;
            const double yj = ssy ? __dadd_rn(pj.y, ssy > 0 ? Ly : -Ly) : pj.y;
            const double zj = ssz ? __dadd_rn(pj.z, ssz > 0 ? Lz : -Lz) : pj.z;
            const double dx = __dsub_rn(pi.x, xj);
            const double dy = __dsub_rn(pi.y, yj);
            const double dz = __dsub_rn(pi.z, zj);
            const double r2 = norm2_rn(dx, dy, dz);
            if (r2 < rc2) {
                if (PREC == 0) {
                    // LJ_accijmag = 48 (s^7 - s^4/2), s = 1/r^2 (setup_set_parameters.f90:105-113)
                    const double s = 1.0 / r2;
                    const double s2 = s * s, s4 = s2 * s2;
                    const double acc = 48.0 * (s4 * s2 * s - 0.5 * s4);
                    fx += acc * dx; fy += acc * dy; fz += acc * dz;
                    if (REC) {
                        const double s3 = s2 * s, s6 = s3 * s3;
                        pe += 4.0 * (s6 - s3) - d.potshift;  // LJ_energy (:126-135)
                        vir += acc * r2;
                    }
                } else {
                    const float s = 1.0f / (float)r2;
                    const float s2 = s * s, s4 = s2 * s2;
                    const float acc = 48.0f * (s4 * s2 * s - 0.5f * s4);
                    fx += (double)(acc * (float)dx);
                    fy += (double)(acc * (float)dy);
                    fz += (double)(acc * (float)dz);
                    if (REC) {
                        const float s3 = s2 * s, s6 = s3 * s3;
                        pe += (double)(4.0f * (s6 - s3)) - d.potshift;
                        vir += (double)(acc * (float)r2);
                    }
                }
            }
        }
    }
    if (TPM > 1) {
#pragma unroll
        for (int o = TPM / 2; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
            if (REC) {
                pe += __shfl_xor_sync(0xffffffffu, pe, o);
                vir += __shfl_xor_sync(0xffffffffu, vir, o);
            }
        }
    }
    double part[RS_N] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double m2 = 0.0;
    if (active && lane == 0) {
        // a(:,i) = sum acc rij / mass, mass = 1 (LJ_mass)
        d.ax[i] = fx; d.ay[i] = fy; d.az[i] = fz;
        if (REC) { d.pe[i] = pe; d.vir[i] = vir; }
        if (MODE >= 1) {
            double vx = __dadd_rn(d.vx[i], __dmul_rn(d.half_dt, fx));
            double vy = __dadd_rn(d.vy[i], __dmul_rn(d.half_dt, fy));
            double vz = __dadd_rn(d.vz[i], __dmul_rn(d.half_dt, fz));
            if (REC) {
                part[RS_PE] = pe;
                part[RS_VIR] = vir;
                part[RS_MV2] = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
                part[RS_VSUM] = __dadd_rn(__dadd_rn(vx, vy), vz);
                part[RS_PEMAX] = pe;
            }
            if (MODE == 2) {
                double4 p = P[i];
                p.x = __dadd_rn(__dadd_rn(p.x, __dmul_rn(d.dt, vx)), __dmul_rn(d.half_dt2, fx));
                p.y = __dadd_rn(__dadd_rn(p.y, __dmul_rn(d.dt, vy)), __dmul_rn(d.half_dt2, fy));
                p.z = __dadd_rn(__dadd_rn(p.z, __dmul_rn(d.dt, vz)), __dmul_rn(d.half_dt2, fz));
                vx = __dadd_rn(vx, __dmul_rn(d.half_dt, fx));
                vy = __dadd_rn(vy, __dmul_rn(d.half_dt, fy));
                vz = __dadd_rn(vz, __dmul_rn(d.half_dt, fz));
                cur_pos(d, pset ^ 1)[i] = p;
                m2 = norm2_rn(vx, vy, vz);
            }
            d.vx[i] = vx; d.vy[i] = vy; d.vz[i] = vz;
        } else if (REC) {
            double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
            part[RS_PE] = pe;
            part[RS_VIR] = vir;
            part[RS_MV2] = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
            part[RS_VSUM] = __dadd_rn(__dadd_rn(vx, vy), vz);
            part[RS_PEMAX] = pe;
        }
    }
    if (REC) block_partials(d, part);
    if (MODE == 2) block_vmax2(d, m2);
}

// Neumaier-compensated reduction of the per-block partials into one record
// (evaluate_macroscopic_properties, simulation_record.f90:1205-1314).
constexpr int REC_THREADS = 256;
__global__ void __launch_bounds__(REC_THREADS) k_record(FmDev d, int iter, double simtime)
{
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
        if (tot[RS_PEMAX] > 10000.0) raise_status(d, ST_PE, iter);
    }
}

// Record partials from per-molecule arrays and current velocities
// (evaluate_macroscopic_properties reads potenergymol, virialmol and v).
constexpr int MACRO_THREADS = 256;
__global__ void __launch_bounds__(MACRO_THREADS) k_macro_partials(FmDev d)
{
    if (frozen(d)) return;
    int i = blockIdx.x * MACRO_THREADS + threadIdx.x;
    double part[RS_N] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < d.n) {
        double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
        part[RS_PE] = d.pe[i];
        part[RS_VIR] = d.vir[i];
        part[RS_MV2] = norm2_rn(vx, vy, vz);
        part[RS_VSUM] = __dadd_rn(__dadd_rn(vx, vy), vz);
        part[RS_PEMAX] = d.pe[i];
    }
    __shared__ double ws[RS_N][MACRO_THREADS / 32];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int k = 0; k < RS_N; k++) {
        double x = k == RS_PEMAX ? warp_max(part[k]) : warp_sum(part[k]);
        if (l == 0) ws[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < RS_N) {
        int k = threadIdx.x;
        double acc = ws[k][0];
        for (int q = 1; q < MACRO_THREADS / 32; q++) acc = k == RS_PEMAX ? fmax(acc, ws[k][q]) : acc + ws[k][q];
        d.partial[(size_t)blockIdx.x * RS_N + k] = acc;
    }
}

// ---------------------------------------------------------------------------
// all pairs with per-axis minimum image (simulation_compute_forces_LJ_AP,
// simulation_compute_forces.f90:280-341), both sides evaluated per molecule
// ---------------------------------------------------------------------------

constexpr int AP_THREADS = 128;
template <bool REC, int MODE, int PREC>
__global__ void __launch_bounds__(AP_THREADS) k_all_pairs(FmDev d)
{
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
                if (r2 < d.rc2) {
                    if (PREC == 0) {
                        const double s = 1.0 / r2;
                        const double s2 = s * s, s4 = s2 * s2;
                        const double acc = 48.0 * (s4 * s2 * s - 0.5 * s4);
                        fx += acc * r[0]; fy += acc * r[1]; fz += acc * r[2];
                        if (REC) {
                            const double s3 = s2 * s, s6 = s3 * s3;
                            pe += 4.0 * (s6 - s3) - d.potshift;
                            vir += acc * r2;
                        }
                    } else {
                        const float s = 1.0f / (float)r2;
                        const float s2 = s * s, s4 = s2 * s2;
                        const float acc = 48.0f * (s4 * s2 * s - 0.5f * s4);
                        fx += (double)(acc * (float)r[0]);
                        fy += (double)(acc * (float)r[1]);
                        fz += (double)(acc * (float)r[2]);
                        if (REC) {
                            const float s3 = s2 * s, s6 = s3 * s3;
                            pe += (double)(4.0f * (s6 - s3)) - d.potshift;
                            vir += (double)(acc * (float)r2);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    double part[RS_N] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double m2 = 0.0;
    if (active) {
        d.ax[i] = fx; d.ay[i] = fy; d.az[i] = fz;
        if (REC) { d.pe[i] = pe; d.vir[i] = vir; }
        double vx = d.vx[i], vy = d.vy[i], vz = d.vz[i];
        if (MODE >= 1) {
            vx = __dadd_rn(vx, __dmul_rn(d.half_dt, fx));
            vy = __dadd_rn(vy, __dmul_rn(d.half_dt, fy));
            vz = __dadd_rn(vz, __dmul_rn(d.half_dt, fz));
        }
        if (REC) {
            part[RS_PE] = pe;
            part[RS_VIR] = vir;
            part[RS_MV2] = norm2_rn(vx, vy, vz);
            part[RS_VSUM] = __dadd_rn(__dadd_rn(vx, vy), vz);
            part[RS_PEMAX] = pe;
        }
        if (MODE == 2) {
            double4 p = pi;
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
    }
    if (REC) {
        // AP blocks are AP_THREADS wide; reuse the generic reduction layout
        __shared__ double ws[RS_N][AP_THREADS / 32];
        int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        for (int k = 0; k < RS_N; k++) {
            double x = k == RS_PEMAX ? warp_max(part[k]) : warp_sum(part[k]);
            if (l == 0) ws[k][w] = x;
        }
        __syncthreads();
        if (threadIdx.x < RS_N) {
            int k = threadIdx.x;
            double acc = ws[k][0];
            for (int q = 1; q < AP_THREADS / 32; q++) acc = k == RS_PEMAX ? fmax(acc, ws[k][q]) : acc + ws[k][q];
            d.partial[(size_t)blockIdx.x * RS_N + k] = acc;
        }
    }
    if (MODE == 2) block_vmax2(d, m2);
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
        const int32_t *L = d.nbr + (size_t)i * d.maxn;
        for (int k = 0; k < d.nnbr[i]; k++) {
            int e = L[k];
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

// upload order u -> slot u (uploads start in upload order)
__global__ void k_scatter_state(FmDev d, const double *r3, const double *v3, const double *a3)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= d.n) return;
    double4 *P = cur_pos(d, d.sc->pset);
    P[u] = make_double4(r3[3 * (size_t)u], r3[3 * (size_t)u + 1], r3[3 * (size_t)u + 2], 0.0);
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
void launch_move1(const FmDev &d, cudaStream_t st) { k_move1<<<nblk(d.n, 256), 256, 0, st>>>(d); }
void launch_move2(const FmDev &d, cudaStream_t st) { k_move2<<<nblk(d.n, 256), 256, 0, st>>>(d); }
void launch_vmax(const FmDev &d, cudaStream_t st) { k_vmax<<<nblk(d.n, 256), 256, 0, st>>>(d); }
void launch_decide(const FmDev &d, int iter, int flip, int crit, int fixed_rebuild, double half_min_delta,
                   cudaStream_t st)
{
    k_decide<<<1, 1, 0, st>>>(d, iter, flip, crit, fixed_rebuild > 0 ? fixed_rebuild : 1, half_min_delta);
}
void launch_wrap_bin(const FmDev &d, int wrap, int bin, int gated, int iter, cudaStream_t st)
{
    k_wrap_bin<<<nblk(d.n, 256), 256, 0, st>>>(d, wrap, bin, gated, iter);
}
void launch_scan_cells(const FmDev &d, int gated, cudaStream_t st) { k_scan_cells<<<1, SCAN_THREADS, 0, st>>>(d, gated); }
void launch_scatter(const FmDev &d, int gated, cudaStream_t st)
{
    k_scatter<<<nblk(d.n, 256), 256, 0, st>>>(d, gated);
    k_sort_cells<<<nblk(d.ncell, 128), 128, 0, st>>>(d, gated);
}
void launch_reorder(const FmDev &d, int gated, double4 *tpos, int32_t *tuidx, cudaStream_t st)
{
    k_reorder_gather<<<nblk(d.n, 256), 256, 0, st>>>(d, gated, tpos, tuidx);
    k_reorder_copy<<<nblk(d.n, 256), 256, 0, st>>>(d, gated, tpos, tuidx);
}
void launch_build_nlist(const FmDev &d, int gated, int iter, cudaStream_t st)
{
    k_build_nlist<<<d.ncell, NB_THREADS, 0, st>>>(d, gated, iter);
}

int force_blocks(int n, int tpm) { return nblk(n * tpm, FORCE_THREADS); }
int all_pairs_blocks(int n) { return nblk(n, AP_THREADS); }

template <int TPM>
static void launch_force_tpm(const FmDev &d, int record, int mode, cudaStream_t st)
{
    const int g = force_blocks(d.n, TPM);
#define FM_FORCE_CASE(R, M)                                                                     \
    if (record == R && mode == M) {                                                             \
        if (d.precision == 0) k_force<TPM, R, M, 0><<<g, FORCE_THREADS, 0, st>>>(d);            \
        else k_force<TPM, R, M, 1><<<g, FORCE_THREADS, 0, st>>>(d);                             \
        return;                                                                                 \
    }
    FM_FORCE_CASE(0, 0) FM_FORCE_CASE(0, 1) FM_FORCE_CASE(0, 2)
    FM_FORCE_CASE(1, 0) FM_FORCE_CASE(1, 1) FM_FORCE_CASE(1, 2)
#undef FM_FORCE_CASE
}

void launch_force(const FmDev &d, int record, int mode, int tpm, cudaStream_t st)
{
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
        if (d.precision == 0) k_all_pairs<R, M, 0><<<g, AP_THREADS, 0, st>>>(d);    \
        else k_all_pairs<R, M, 1><<<g, AP_THREADS, 0, st>>>(d);                     \
        return;                                                                     \
    }
    FM_AP_CASE(0, 0) FM_AP_CASE(0, 1) FM_AP_CASE(0, 2)
    FM_AP_CASE(1, 0) FM_AP_CASE(1, 1) FM_AP_CASE(1, 2)
#undef FM_AP_CASE
}

int macro_blocks(int n) { return nblk(n, MACRO_THREADS); }
void launch_macro_partials(const FmDev &d, cudaStream_t st)
{
    k_macro_partials<<<macro_blocks(d.n), MACRO_THREADS, 0, st>>>(d);
}

void launch_record(const FmDev &d, int iter, double simtime, cudaStream_t st)
{
    k_record<<<1, REC_THREADS, 0, st>>>(d, iter, simtime);
}

void launch_pair_digest(const FmDev &d, const int32_t *glob_of_upload, cudaStream_t st)
{
    k_pair_digest<<<nblk(d.n, 256), 256, 0, st>>>(d, glob_of_upload);
}

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
