// fm_sort.cu -- sort_mols (linklist.f90:2744-2869) for a single system.
//
// Every sort_freq rebuilds the reference re-orders its molecule arrays r, v
// (and tag, rtether): each molecule goes to the block of sortblocksize^3
// cells that holds it, blocks are taken in the order of the table Hcurve
// (setup_set_parameters.f90:1140-1163: x-fastest block numbers for
// sort_flag 1, a 3-D Hilbert curve for 2), and molecules keep their relative
// order inside a block.  If a block holds more than ave_molperblock molecules
// the sort is skipped and the safety factors grow.
//
// The device keeps its molecules in cell order whatever the caller's order,
// so here the sort changes the caller's numbering: the upload index of every
// molecule (slot_of, by which downloads scatter) and the global numbers kept
// by upload index.  The new upload order is the reference's new array order.
// The next cell sort orders each cell's members by that numbering, so the
// list order and the FP64 summation order follow it as the reference's
// follow its array order.
//
// Device steps, inside the rebuild branch after the periodic wrap and before
// the cell counting sort (all gated: they exit unless this step rebuilds and
// the counter says sort):
//   k_sort_gate   the rebuild counter nrebuilds and ave_molperblock
//   k_sort_keys   block of each molecule by upload index, block counts and
//                 the overflow flag
//   radix sort    (block, upload index) pairs: stable, so the molecules of a
//                 block keep their order (CUB DeviceRadixSort, library code;
//                 its size is fixed at launch, so it cannot return early: in
//                 the step graphs it sits with the kernels below in a nested
//                 conditional node that k_sort_gate_graph opens only on the
//                 rebuilds that sort; launched one by one it runs whenever
//                 the gate does)
//   k_sort_rank   new upload index of every old one; block counts cleared for
//                 the next sort; an overflow grows the safety factors instead
//   k_sort_apply  slot_of renumbered, global numbers permuted into scratch
//   k_sort_copy   scratch back into the global numbers
#include "fm_common.cuh"
#include "flowmol_b200.h"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

namespace fm {
namespace {

__device__ __forceinline__ bool sort_gate(const FmDev &d, int gated)
{
    if ((d.sc->status & ST_FATAL) != 0u) return false;
    return !gated || d.sc->rebuild;
}

// ceiling((r + halfdomain) / blocksidelength) (linklist.f90:2815-2817),
// rounded as the reference rounds it: one add, one divide.
__device__ __forceinline__ int sort_block(double r, double hd, double bsl)
{
    return (int)ceil(__ddiv_rn(__dadd_rn(r, hd), bsl));
}

// The rebuild counter (linklist.f90:2766-2771) and ave_molperblock =
// ceiling((np/blocks)*sf1 + sf2) (:2794-2796: an integer quotient, then one
// multiply and one add in FP64).  Returns whether this rebuild sorts.
__device__ bool sort_due(const FmDev &d, const FmSortDev &s)
{
    FmSortScalars &q = *s.ss;
    q.due = 0;
    if (q.nrebuilds != s.freq) {
        q.nrebuilds += 1;
        return false;
    }
    q.nrebuilds = 1;
    const int ave = d.n / s.blocks;
    q.ave = (int)ceil(__dadd_rn(__dmul_rn((double)ave, q.sf1), (double)q.sf2));
    q.overflow = 0;
    q.due = 1;
    return true;
}

__global__ void k_sort_gate(FmDev d, FmSortDev s, int gated)
{
    if (threadIdx.x != 0 || !sort_gate(d, gated)) return;
    sort_due(d, s);
}

// In the rebuild graph's body: opens the nested conditional node that holds
// the rest of the sort only when this rebuild sorts (the condition's default
// is 0 at every graph launch), and counts the kernels the node will run.
__global__ void k_sort_gate_graph(FmDev d, FmSortDev s, cudaGraphConditionalHandle cond, int body_kernels)
{
    if (threadIdx.x != 0 || !sort_gate(d, 1)) return;
    if (sort_due(d, s)) {
        d.sc->graph_kernels += body_kernels;
        cudaGraphSetConditional(cond, 1u);
    }
}

__global__ void k_sort_keys(FmDev d, FmSortDev s, int gated)
{
    if (!sort_gate(d, gated) || !s.ss->due) return;
    const double4 *P = cur_pos(d, d.sc->pset);
    const int ave = s.ss->ave;
    const long long last = (long long)s.blocks - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += gridDim.x * blockDim.x) {
        const double4 p = P[i];
        const int ib = sort_block(p.x, d.hd[0], s.bsl[0]);
        const int jb = sort_block(p.y, d.hd[1], s.bsl[1]);
        const int kb = sort_block(p.z, d.hd[2], s.bsl[2]);
        // Hcurve(iblk, jblk, kblk) by its column-major offset.  A molecule on
        // the lower face (r = -halfdomain) gets block 0, outside the table;
        // the reference then reads the neighbouring element of its array
        // (no bounds checks), which the offset reproduces, and the two ends
        // are clamped.
        long long lin = (long long)(ib - 1) + (long long)s.nb[0] * ((long long)(jb - 1) + (long long)s.nb[1] * (kb - 1));
        lin = lin < 0 ? 0 : (lin > last ? last : lin);
        const int key = s.hc[lin] - 1;
        s.key[d.slot_of[i]] = key;
        if (atomicAdd(&s.cnt[key], 1) + 1 > ave) s.ss->overflow = 1;  // :2822-2829
    }
}

__global__ void k_sort_rank(FmDev d, FmSortDev s, int gated)
{
    if (!sort_gate(d, gated) || !s.ss->due) return;
    const bool overflow = s.ss->overflow != 0;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (!overflow)
        for (int p = tid; p < d.n; p += stride) s.newv[s.val_out[p]] = p;
    for (int b = tid; b < s.blocks; b += stride) s.cnt[b] = 0;
    if (tid == 0) {
        FmSortScalars &q = *s.ss;
        if (overflow) {  // sf1 = sf1 + 0.1d0; sf2 = sf2 + 5 (:2824)
            q.sf1 = __dadd_rn(q.sf1, 0.1);
            q.sf2 += 5;
            q.skipped += 1;
        } else {
            q.sorts += 1;
        }
    }
}

__global__ void k_sort_apply(FmDev d, FmSortDev s, int gated)
{
    if (!sort_gate(d, gated) || !s.ss->due || s.ss->overflow) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += gridDim.x * blockDim.x) {
        d.slot_of[i] = s.newv[d.slot_of[i]];
        s.gtmp[s.newv[i]] = s.glob[i];
    }
}

__global__ void k_sort_copy(FmDev d, FmSortDev s, int gated)
{
    if (!sort_gate(d, gated) || !s.ss->due || s.ss->overflow) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += gridDim.x * blockDim.x)
        s.glob[i] = s.gtmp[i];
}

int grid_for(int n)
{
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, std::min((n + 255) / 256, nsm * 8));
}

// One point of the level-h Hilbert curve of build_hilbert's hilbert3
// (functions_lib.f90:2609-2637).  Level l maps the level l-1 curve into the
// eight octants, copy k for the k-th eighth of the points, so point i is the
// origin carried through the octant maps of its base-8 digits, lowest first.
// Each map is one of the eight coordinate patterns below; every value is a
// dyadic fraction, exact in FP64.
void hilbert_point(long long i, int h, double &x, double &y, double &z)
{
    x = y = z = 0.0;
    for (int l = 0; l < h; l++) {
        const int k = (int)((i >> (3 * l)) & 7);
        const double xo = x, yo = y, zo = z;
        switch (k) {
        case 0: x = 0.5 * (0.5 + zo); y = 0.5 * (0.5 + xo); z = 0.5 * (0.5 + yo); break;
        case 1: x = 0.5 * (0.5 + yo); y = 0.5 * (0.5 + zo); z = 0.5 * (-0.5 + xo); break;
        case 2: x = 0.5 * (-0.5 + yo); y = 0.5 * (0.5 + zo); z = 0.5 * (-0.5 + xo); break;
        case 3: x = 0.5 * (-0.5 - xo); y = 0.5 * (0.5 + yo); z = 0.5 * (0.5 - zo); break;
        case 4: x = 0.5 * (-0.5 - xo); y = 0.5 * (-0.5 + yo); z = 0.5 * (0.5 - zo); break;
        case 5: x = 0.5 * (-0.5 - yo); y = 0.5 * (-0.5 - zo); z = 0.5 * (-0.5 + xo); break;
        case 6: x = 0.5 * (0.5 - yo); y = 0.5 * (-0.5 - zo); z = 0.5 * (-0.5 + xo); break;
        default: x = 0.5 * (0.5 + zo); y = 0.5 * (-0.5 - xo); z = 0.5 * (0.5 - yo); break;
        }
    }
}

}  // namespace

// Curves above 2^10 blocks per axis (8^10 points) are refused.
constexpr int SORT_MAX_LEVEL = 10;

int sort_table(int flag, const int nb[3], int32_t *out, const char **why)
{
    const long long blocks = (long long)nb[0] * nb[1] * nb[2];
    if (nb[0] < 1 || nb[1] < 1 || nb[2] < 1) { *why = "sort blocks per axis must be positive"; return -1; }
    if (flag == 1) {  // setup_set_parameters.f90:1143-1155
        for (int k = 0; k < nb[2]; k++)
            for (int j = 0; j < nb[1]; j++)
                for (int i = 0; i < nb[0]; i++) {
                    const long long lin = i + (long long)nb[0] * (j + (long long)nb[1] * k);
                    out[lin] = (int32_t)(lin + 1);
                }
        return 0;
    }
    if (flag != 2) { *why = "Incorrect value of sort_flag"; return -1; }
    // build_hilbert (functions_lib.f90:2555-2604): the level is the ceiling of
    // log2 of the longest axis, taken through the natural log as the
    // reference does; for a longest axis that is not a power of two the grid
    // the curve is scaled to is ceiling(8**(h/3)), which the FP64 pow rounds
    // to 2^h + 1 for some h (the curve's points still land on cells 1..2^h)
    int maxc = std::max(nb[0], std::max(nb[1], nb[2]));
    const double l2 = std::log((double)maxc) / std::log(2.0);
    const int h = (int)std::ceil(l2);
    if (h > SORT_MAX_LEVEL) { *why = "Hilbert sort above 1024 blocks per axis"; return -1; }
    if ((double)h - l2 > 0.0001) maxc = (int)std::ceil(std::pow(8.0, (double)h / 3.0));
    const long long npts = 1ll << (3 * h);
    double lo = 0.0;
    for (long long i = 0; i < npts; i++) {
        double x, y, z;
        hilbert_point(i, h, x, y, z);
        lo = std::min(lo, std::min(x, std::min(y, z)));
    }
    const double shift = 0.00001 - lo;
    std::fill(out, out + blocks, -666);
    int32_t m = 0;
    for (long long i = 0; i < npts; i++) {
        double x, y, z;
        hilbert_point(i, h, x, y, z);
        const int ic = (int)std::ceil((x + shift) * (double)maxc);
        const int jc = (int)std::ceil((y + shift) * (double)maxc);
        const int kc = (int)std::ceil((z + shift) * (double)maxc);
        if (ic <= nb[0] && jc <= nb[1] && kc <= nb[2]) {
            m += 1;
            out[(ic - 1) + (long long)nb[0] * ((jc - 1) + (long long)nb[1] * (kc - 1))] = m;
        }
    }
    for (long long b = 0; b < blocks; b++)
        if (out[b] == -666) { *why = "Error in generating Hilbert curve - change sort flag"; return -1; }
    // the reference counts molecules per block at molperblock(Hcurve value):
    // a curve that visited a cell twice would index past its blocks
    if (m > blocks) { *why = "Hilbert curve numbers exceed the blocks"; return -1; }
    return 0;
}

size_t sort_scratch_bytes(int n, int end_bit)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const int32_t *)nullptr, (int32_t *)nullptr,
                                    (const int32_t *)nullptr, (int32_t *)nullptr, n, 0, end_bit);
    return bytes;
}

void launch_sort_body(const FmDev &d, const FmSortDev &s, int gated, cudaStream_t st)
{
    const int g = grid_for(std::max(d.n, s.blocks));
    k_sort_keys<<<g, 256, 0, st>>>(d, s, gated);
    size_t bytes = s.tmp_bytes;
    cub::DeviceRadixSort::SortPairs(s.tmp, bytes, s.key, s.key_out, s.val, s.val_out, d.n, 0, s.end_bit, st);
    k_sort_rank<<<g, 256, 0, st>>>(d, s, gated);
    k_sort_apply<<<g, 256, 0, st>>>(d, s, gated);
    k_sort_copy<<<g, 256, 0, st>>>(d, s, gated);
}

void launch_sort(const FmDev &d, const FmSortDev &s, int gated, cudaStream_t st)
{
    k_sort_gate<<<1, 32, 0, st>>>(d, s, gated);
    launch_sort_body(d, s, gated, st);
}

void launch_sort_gate_graph(const FmDev &d, const FmSortDev &s, cudaGraphConditionalHandle cond, int body_kernels,
                            cudaStream_t st)
{
    k_sort_gate_graph<<<1, 32, 0, st>>>(d, s, cond, body_kernels);
}

}  // namespace fm

// Hcurve for a grid of sort blocks: the table sort_mols orders blocks by
// (setup_set_parameters.f90:1140-1163, functions_lib.f90:2555-2604).
extern "C" int fm_sort_table(int32_t sort_flag, const int32_t nblocks[3], int32_t *table, int64_t cap)
{
    if (!nblocks || !table) {
        fm::set_last_error("null argument");
        return FM_ERR_ARG;
    }
    const int nb[3] = {nblocks[0], nblocks[1], nblocks[2]};
    if (nb[0] < 1 || nb[1] < 1 || nb[2] < 1 || (long long)nb[0] * nb[1] * nb[2] > cap) {
        fm::set_last_error("sort blocks must be positive and fit in cap");
        return FM_ERR_ARG;
    }
    const char *why = nullptr;
    if (fm::sort_table(sort_flag, nb, table, &why) != 0) {
        fm::set_last_error(why);
        return FM_ERR_ARG;
    }
    return FM_OK;
}
