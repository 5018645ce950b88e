// fm_dd_kernels.cu -- device side of the spatial decomposition: one rank's
// subdomain of the cell grid (messenger.MPI.f90:222-550), its molecule
// migration on rebuilds (sendmols, :1383-1421) and its halo of copies of the
// neighbouring subdomains' boundary cells (messenger_updateborders,
// :594-628, faces/edges/corners :882-1380).
//
// Unlike the reference, which gives every rank local coordinates and its own
// cell count, a subdomain here keeps global coordinates and a block of the
// undivided system's cells (interior cells org .. org + nc - 1 per axis).  A
// molecule is binned with the undivided system's formula and its owner is
// the rank holding that cell, so the ranks' cells, the molecules in them and
// their order (by global number) are the undivided system's, and so are the
// neighbour rows and every force bit.  The exchanges themselves (counts, then
// records, rank to rank) are the caller's (NCCL or gloo all-to-all); these
// kernels fill and drain the flat record buffers.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fm_common.cuh"
#include "fm_device.cuh"

namespace fm {

namespace {

__device__ __forceinline__ void dd_raise(const FmDev &d, uint32_t bit, int iter)
{
    if (atomicOr(&d.sc->status, bit) == 0u) d.sc->fail_iter = iter;
}

// Owner rank and this rank's local extended cell (-1 when not this rank's) of
// a global position; false when it bins outside the global interior.
__device__ __forceinline__ bool dd_locate(const FmDev &d, const DdDev &x, double4 p, int &owner, int &cell)
{
    bool bad = false;
    const int gx = bin_axis(p.x, d.hd[0], d.cs[0], d.gne[0], bad);
    const int gy = bin_axis(p.y, d.hd[1], d.cs[1], d.gne[1], bad);
    const int gz = bin_axis(p.z, d.hd[2], d.cs[2], d.gne[2], bad);
    // the global halo layer (a molecule exactly on the lower box face, the
    // reference's ceiling quirk) has no owner here
    if (bad || gx == 0 || gy == 0 || gz == 0 || gx == d.gne[0] - 1 || gy == d.gne[1] - 1 || gz == d.gne[2] - 1)
        return false;
    const int G0 = d.gne[0] - 2, G1 = d.gne[1] - 2;
    const int px = x.owner_axis[gx - 1], py = x.owner_axis[G0 + gy - 1], pz = x.owner_axis[G0 + G1 + gz - 1];
    owner = (px * x.dims[1] + py) * x.dims[2] + pz;
    cell = -1;
    if (owner == x.rank) {
        const int lx = gx - d.org[0], ly = gy - d.org[1], lz = gz - d.org[2];
        cell = lx + d.ne[0] * (ly + d.ne[1] * lz);
    }
    return true;
}

// Classifies the molecules [0, n): halo copies are dropped (cell_of = -1);
// owned molecules are wrapped into the box (sendmols' periodic wrap, when
// `wrap`), binned and either kept (cell_of, cell_count) or listed as
// emigrants with their destination (per-destination counts).
__global__ void k_dd_classify(FmDev d, DdDev x, int n, int wrap, int iter)
{
    double4 *P = cur_pos(d, d.sc->pset);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double4 p = P[i];
        if (p.w != 0.0) { d.cell_of[i] = -1; continue; }
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
        int owner = 0, cell = -1;
        if (!dd_locate(d, x, p, owner, cell)) {
            dd_raise(d, ST_ESCAPE, iter);
            d.sc->escape_slot = i;
            d.cell_of[i] = -1;
            continue;
        }
        if (cell >= 0) {
            d.cell_of[i] = cell;
            atomicAdd(&d.cell_count[cell], 1);
            continue;
        }
        d.cell_of[i] = -1;
        atomicAdd(&x.count[owner], 1);
        const int k = atomicAdd(x.nlist, 1);
        if (k < x.list_cap) {
            x.list_idx[k] = i;
            x.list_aux[k] = owner;
        } else {
            dd_raise(d, ST_MIGRATE, iter);
        }
    }
}

// Emigrant records (DD_MREC doubles: r, v, a, global number) grouped by
// destination at the host's offsets.
__global__ void k_dd_pack_emigrants(FmDev d, DdDev x, double *out)
{
    const double4 *P = cur_pos(d, d.sc->pset);
    const int n = min(*x.nlist, x.list_cap);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = x.list_idx[k], dest = x.list_aux[k];
        const int pos = x.offset[dest] + atomicAdd(&x.cursor[dest], 1);
        double *r = out + (size_t)pos * DD_MREC;
        const double4 p = P[i];
        r[0] = p.x; r[1] = p.y; r[2] = p.z;
        r[3] = d.vx[i]; r[4] = d.vy[i]; r[5] = d.vz[i];
        r[6] = d.ax[i]; r[7] = d.ay[i]; r[8] = d.az[i];
        r[9] = (double)d.slot_of[i];
    }
}

// Immigrant records appended at [base, base + n): binned into this rank's
// cells (a molecule that does not bin here raises ST_MIGRATE).
__global__ void k_dd_append_immigrants(FmDev d, DdDev x, const double *in, int n, int base, int iter)
{
    double4 *P = cur_pos(d, d.sc->pset);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double *r = in + (size_t)k * DD_MREC;
        const int i = base + k;
        const double4 p = make_double4(r[0], r[1], r[2], 0.0);
        P[i] = p;
        d.vx[i] = r[3]; d.vy[i] = r[4]; d.vz[i] = r[5];
        d.ax[i] = r[6]; d.ay[i] = r[7]; d.az[i] = r[8];
        d.slot_of[i] = (int32_t)r[9];
        int owner = 0, cell = -1;
        if (!dd_locate(d, x, p, owner, cell) || cell < 0) {
            dd_raise(d, ST_MIGRATE, iter);
            d.cell_of[i] = -1;
            continue;
        }
        d.cell_of[i] = cell;
        atomicAdd(&d.cell_count[cell], 1);
    }
}

// Halo records of the kept molecules [0, n): one per (molecule, need of its
// cell) -- a need is a neighbouring rank whose halo holds this cell, the
// periodic shift it sees the cell with and the local halo cell there.
// Pass 0 counts per destination; pass 1 writes records (DD_HREC doubles:
// shifted r, global number, destination cell) at the host's offsets.
__global__ void k_dd_halo_records(FmDev d, DdDev x, int n, int pass, double *out)
{
    const double4 *P = cur_pos(d, d.sc->pset);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = d.cell_of[i];
        if (c < 0) continue;
        const int k0 = x.need_off[c], k1 = x.need_off[c + 1];
        if (k0 == k1) continue;
        const double4 p = P[i];
        for (int k = k0; k < k1; k++) {
            const int dest = x.need_rank[k];
            if (pass == 0) { atomicAdd(&x.count[dest], 1); continue; }
            const int code = x.need_code[k];
            const int pos = x.offset[dest] + atomicAdd(&x.cursor[dest], 1);
            double *r = out + (size_t)pos * DD_HREC;
            r[0] = image(p.x, (code & 3) - 1, d.L[0]);
            r[1] = image(p.y, ((code >> 2) & 3) - 1, d.L[1]);
            r[2] = image(p.z, ((code >> 4) & 3) - 1, d.L[2]);
            r[3] = (double)d.slot_of[i];
            r[4] = (double)x.need_cell[k];
        }
    }
}

// Halo copies appended at [base, base + n) into their halo cells: w = 1,
// v = a = 0 (they feel no force and never move), no rows.
__global__ void k_dd_append_halo(FmDev d, const double *in, int n, int base)
{
    double4 *P = cur_pos(d, d.sc->pset);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double *r = in + (size_t)k * DD_HREC;
        const int i = base + k;
        P[i] = make_double4(r[0], r[1], r[2], 1.0);
        d.vx[i] = 0.0; d.vy[i] = 0.0; d.vz[i] = 0.0;
        d.ax[i] = 0.0; d.ay[i] = 0.0; d.az[i] = 0.0;
        d.slot_of[i] = (int32_t)r[3];
        const int c = (int)r[4];
        d.cell_of[i] = c;
        atomicAdd(&d.cell_count[c], 1);
    }
}

// Per-step halo refresh: positions of the listed molecules, shifted by their
// image code, into a flat (x, y, z) buffer; and the receiving side's copy
// into its halo slots.
__global__ void k_dd_gather_positions(FmDev d, const int32_t *idx, const int8_t *code, int n, double *out)
{
    const double4 *P = cur_pos(d, d.sc->pset);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double4 p = P[idx[k]];
        const int c = code[k];
        out[3 * (size_t)k] = image(p.x, (c & 3) - 1, d.L[0]);
        out[3 * (size_t)k + 1] = image(p.y, ((c >> 2) & 3) - 1, d.L[1]);
        out[3 * (size_t)k + 2] = image(p.z, ((c >> 4) & 3) - 1, d.L[2]);
    }
}

__global__ void k_dd_scatter_positions(FmDev d, const int32_t *idx, const double *in, int n)
{
    double4 *P = cur_pos(d, d.sc->pset);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = idx[k];
        P[i] = make_double4(in[3 * (size_t)k], in[3 * (size_t)k + 1], in[3 * (size_t)k + 2], 1.0);
    }
}

// Neumaier totals of the record partials of the last record step (the sums
// evaluate_macroscopic_properties forms; the ranks' totals are summed by the
// caller): out[RS_N].
constexpr int DS_THREADS = 256;
__global__ void __launch_bounds__(DS_THREADS) k_dd_sums(FmDev d, double *out)
{
    __shared__ double ssum[RS_N][DS_THREADS], scmp[RS_N][DS_THREADS];
    double sum[RS_N], cmp[RS_N];
    for (int k = 0; k < RS_N; k++) { sum[k] = 0.0; cmp[k] = 0.0; }
    for (int b = threadIdx.x; b < d.nblocks_force; b += DS_THREADS) {
        for (int k = 0; k < RS_N; k++) {
            const double v = d.partial[(size_t)b * RS_N + k];
            if (k == RS_PEMAX) { sum[k] = fmax(sum[k], v); continue; }
            neumaier(sum[k], cmp[k], v);
        }
    }
    for (int k = 0; k < RS_N; k++) { ssum[k][threadIdx.x] = sum[k]; scmp[k][threadIdx.x] = cmp[k]; }
    __syncthreads();
    if (threadIdx.x < RS_N) {
        const int k = threadIdx.x;
        double s = 0.0, c = 0.0;
        for (int q = 0; q < DS_THREADS; q++) {
            if (k == RS_PEMAX) { s = fmax(s, ssum[k][q]); continue; }
            neumaier(s, c, ssum[k][q]);
            c += scmp[k][q];
        }
        out[k] = k == RS_PEMAX ? s : s + c;
    }
}

inline int dd_grid(int n, int t) { return std::max(1, std::min((n + t - 1) / t, 148 * 8)); }

}  // namespace

void launch_dd_classify(const FmDev &d, const DdDev &x, int n, int wrap, int iter, cudaStream_t st)
{
    if (n > 0) k_dd_classify<<<dd_grid(n, 256), 256, 0, st>>>(d, x, n, wrap, iter);
}
void launch_dd_pack_emigrants(const FmDev &d, const DdDev &x, int n, double *out, cudaStream_t st)
{
    if (n > 0) k_dd_pack_emigrants<<<dd_grid(n, 256), 256, 0, st>>>(d, x, out);
}
void launch_dd_append_immigrants(const FmDev &d, const DdDev &x, const double *in, int n, int base, int iter,
                                 cudaStream_t st)
{
    if (n > 0) k_dd_append_immigrants<<<dd_grid(n, 256), 256, 0, st>>>(d, x, in, n, base, iter);
}
void launch_dd_halo_records(const FmDev &d, const DdDev &x, int n, int pass, double *out, cudaStream_t st)
{
    if (n > 0) k_dd_halo_records<<<dd_grid(n, 256), 256, 0, st>>>(d, x, n, pass, out);
}
void launch_dd_append_halo(const FmDev &d, const double *in, int n, int base, cudaStream_t st)
{
    if (n > 0) k_dd_append_halo<<<dd_grid(n, 256), 256, 0, st>>>(d, in, n, base);
}
void launch_dd_gather_positions(const FmDev &d, const int32_t *idx, const int8_t *code, int n, double *out,
                                cudaStream_t st)
{
    if (n > 0) k_dd_gather_positions<<<dd_grid(n, 256), 256, 0, st>>>(d, idx, code, n, out);
}
void launch_dd_scatter_positions(const FmDev &d, const int32_t *idx, const double *in, int n, cudaStream_t st)
{
    if (n > 0) k_dd_scatter_positions<<<dd_grid(n, 256), 256, 0, st>>>(d, idx, in, n);
}
void launch_dd_sums(const FmDev &d, double *out, cudaStream_t st)
{
    k_dd_sums<<<1, DS_THREADS, 0, st>>>(d, out);
}

}  // namespace fm
