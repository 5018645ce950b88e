// fm_build.cuh -- the neighbour-list build of one cell, shared by the
// single-system kernel (fm_kernels.cu) and the slot engine
// (fm_engine_kernels.cu).
//
// Pair set of assign_to_neighbourlist_halfint_opt (linklist.f90:660-804,
// 1118-1180), stored for both partners.  The reference visits every pair of
// adjacent cells of which at least one is interior exactly once (13 forward
// shifts from interior cells + 27 sweeps from halo cells); a halo cell holds
// the images of the interior cell on the far side (plus any real molecule
// that binned onto it).  Here each molecule of cell c collects, from the 27
// cells around c that are not both halo with c, every candidate with
// r^2 < rneighbr^2 -- the same set.
//
// Lane q < 27 computes the segments of neighbour cell q (its real members and,
// for a halo cell, the shifted images of its source); a warp prefix sum lays
// the candidates out in the reference's visiting order (cell q ascending,
// real before images, slot ascending).  Candidates are staged in shared
// memory as FP32 offsets from the cell's reference point, computed from the
// FP64 image coordinate (x_src +/- L, one rounding, as the halo copy); those
// farther than rneighbr from the bounding box of the owners being processed
// are dropped at staging (the order of the rest is kept).  Then each lane
// takes one staged candidate and the warp loops over the owners, NB_OG at a
// time: the FP32 r^2 (error below 1e-5 cs^2 for molecules binned in this
// build, offsets within 1.5 cells) decides every candidate farther than
// BAND = 1e-4 cs^2 from rneighbr2; a candidate inside the band is re-read in
// FP64 and decided by the exact test (dx^2+dy^2)+dz^2 < rneighbr2 -- a branch
// the whole warp skips unless some lane needs it.  An owner's hits among 32
// candidates are one ballot; the owner's lane appends them to its row in
// candidate order (all but its own entry, at distance 0), so every row lists
// its partners in the visiting order.
//
// With FENE polymers (POLY) the same scan discovers bonds the way the
// reference's check_update_adjacentbeadinfo does (linklist.f90:2542-2584): any
// candidate of the scanned cells -- at any distance -- with the owner's chain
// whose subchain bit is set in the owner's bin_bflag words (get_bondflag,
// modules.f90:602-610, 31 bits per word) is a bond partner.  Pruning is off
// then (a stretched bond is still found, and fails at the force).
//
// With TILE the rows hold, instead of the entry bits, the candidate's 16-bit
// word offset in the tiled force kernel's staging of the owner's block
// (fm_tile.cuh): the segment's base in that staging (blk_off) plus the
// candidate's place in its segment.  The pair set and the row order are the
// same.
#pragma once
#include "fm_common.cuh"
#include "fm_device.cuh"
#include "fm_tile.cuh"

namespace fm {

constexpr int NB_WARPS = 4;                 // cells processed concurrently per block
constexpr int NB_THREADS = 32 * NB_WARPS;
constexpr int NB_STAGE = 256;               // staged candidates per warp
constexpr int NB_OG = 4;                    // owners per step of the candidate loop
constexpr int NB_CHUNK = 2;                 // work units a warp takes per fetch (one system)
constexpr int NB_NOSHIFT = 1 | (1 << 2) | (1 << 4);

// One periodic system as the build sees it.  Molecule indices in entries,
// rows and the per-molecule arrays count from the system's first molecule;
// cell_start holds arena indices, mol_off is subtracted from them.
struct CellSys {
    const double4 *P;           // positions of the system's molecules
    const int32_t *cell_start;  // ncell + 1 starts (arena molecule indices)
    int mol_off;
    int ne[3];
    double cs[3], hd[3], L[3];
    double rn2;
    int32_t *nbr;               // rows nb_row(i, maxn) + nb_col(k)
    int32_t *nnbr;
    int maxn;
    int *max_nbr;               // atomicMax of the row lengths
    // FENE (POLY only)
    const int32_t *chain, *subchain;
    const int4 *bflag;
    int32_t *bnd, *nbond;
    // tiled force path (TILE only): rows of staging offsets
    uint16_t *nbr16;
    int maxn16, tT, tR;
    int tdummy;                 // byte offset of the staging's dummy candidate (row padding)
    const int32_t *blk_off;
    int tnb[3];
    // subdomain (dd = 1): halo cells hold explicit copies (no images, no
    // rows); cell x of this grid is global extended cell x + org[0]
    int dd;
    int org[3];
};

// Per-warp shared staging.
template <bool POLY, bool TILE = false>
struct BuildShared {
    float4 f[NB_STAGE];         // x, y, z offsets and the entry bits in w
    alignas(16) float ox[32];   // owners' offsets (+1e30 past the last owner),
    alignas(16) float oy[32];   // read in 8-byte pairs
    alignas(16) float oz[32];
    int oi[32];                 // owners' molecule indices
    int2 cs[POLY ? NB_STAGE : 1];  // chain, subchain of candidates
    int off[55];                // candidate offset of segment k (54 segments + total)
    int start[54], code[54];
    int lbase[TILE ? 54 : 1];                   // segment k's first candidate in the block staging
    unsigned short loc[TILE ? NB_STAGE : 1];    // staged candidates' staging offsets
    alignas(16) int ob[TILE ? 1 : 32][8];       // owner lane's chunk being filled (generic rows)
    alignas(16) unsigned short ob16[TILE ? 32 : 1][32];  // (tiled rows, 4 T <= 32 entries)
    int ochain[POLY ? 32 : 1];
    alignas(16) int4 obf[POLY ? 32 : 1];
    unsigned hits[POLY ? 1 : 32];  // per owner: which of the 32 candidates hit (polymers: registers)
};

constexpr uint32_t BUILD_OVER_LIST = 1u, BUILD_OVER_BONDS = 2u;

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two owners' distance terms
// per instruction, each half rounded exactly as the scalar operation.
__device__ __forceinline__ unsigned long long pack_f32x2(float lo, float hi)
{
    return (unsigned long long)__float_as_uint(lo) | ((unsigned long long)__float_as_uint(hi) << 32);
}
__device__ __forceinline__ unsigned long long lds_f32x2(const float *p)  // 8-byte aligned
{
    return *reinterpret_cast<const unsigned long long *>(p);
}
__device__ __forceinline__ unsigned long long sub_f32x2(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long mul_f32x2(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long fma_f32x2(unsigned long long a, unsigned long long b,
                                                        unsigned long long c)
{
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Exact FP64 decision of a staged candidate (entry e) for owner io: not the
// owner itself, and (dx^2+dy^2)+dz^2 < rneighbr2 with the image x_src +/- L.
__device__ __forceinline__ bool exact_pair(const double4 *P, int io, int e, const double (&L)[3], double rn2)
{
    const int code = e >> NB_SHIFT_BITS, jj = e & NB_INDEX_MASK;
    if (jj == io && code == NB_NOSHIFT) return false;
    const double4 po = ldg_pos(P + io);
    const double4 pj = ldg_pos(P + jj);
    const double xj = image(pj.x, (code & 3) - 1, L[0]);
    const double yj = image(pj.y, ((code >> 2) & 3) - 1, L[1]);
    const double zj = image(pj.z, ((code >> 4) & 3) - 1, L[2]);
    return norm2_rn(__dsub_rn(po.x, xj), __dsub_rn(po.y, yj), __dsub_rn(po.z, zj)) < rn2;
}

// Appends entry cnt (< maxn) of the owner (slot i) of this lane: into the
// lane's chunk buffer, and the chunk to the row once it is full, so that every
// sector of the row is written whole.  Generic rows: a chunk is 8 entries
// (32 bytes) at nb_col(8c).  Tiled rows: a chunk is the 4 T entries of one load
// of the owner's T lanes, contiguous at tile_pos16(4Tc), entry k at place
// (k % T) 4 + (k / T) % 4 of it.
template <bool TILE, typename SH>
__device__ __forceinline__ void append_entry(SH &sh, int lane, int T, int32_t *nbr, uint16_t *row16, int i,
                                             int maxn, int cnt, int ent, unsigned short loc)
{
    if (TILE) {
        const int ch = 4 * T, k = cnt % ch;
        sh.ob16[lane][(k % T) * 4 + (k / T) % 4] = loc;
        if (k == ch - 1) {
            const uint4 *src = reinterpret_cast<const uint4 *>(sh.ob16[lane]);
            uint4 *dst = reinterpret_cast<uint4 *>(row16 + (cnt - k));
            for (int q = 0; q < ch / 8; q++) dst[q] = src[q];
        }
    } else {
        sh.ob[lane][cnt & 7] = ent;
        if ((cnt & 7) == 7) {
            const int4 *src = reinterpret_cast<const int4 *>(sh.ob[lane]);
            int4 *dst = reinterpret_cast<int4 *>(nbr + nb_row(i, maxn) + nb_col(cnt & ~7));
            dst[0] = src[0];
            dst[1] = src[1];
        }
    }
}

// Writes the owner's last, partial chunk (cnt entries in all, cnt < maxn; the
// chunk lies inside the row because maxn is a whole number of chunks).  Tiled
// rows are padded with the dummy candidate up to the chunk's end, the force
// kernel's last load; generic rows leave the places past cnt unread.
template <bool TILE, typename SH>
__device__ __forceinline__ void flush_entries(SH &sh, int lane, int T, int32_t *nbr, uint16_t *row16, int i,
                                              int maxn, int cnt, int dummy)
{
    if (TILE) {
        const int ch = 4 * T, k0 = cnt % ch;
        if (k0 == 0) return;
        for (int k = k0; k < ch; k++) sh.ob16[lane][(k % T) * 4 + (k / T) % 4] = (unsigned short)dummy;
        const uint4 *src = reinterpret_cast<const uint4 *>(sh.ob16[lane]);
        uint4 *dst = reinterpret_cast<uint4 *>(row16 + (cnt - k0));
        for (int q = 0; q < ch / 8; q++) dst[q] = src[q];
    } else {
        if ((cnt & 7) == 0) return;
        const int4 *src = reinterpret_cast<const int4 *>(sh.ob[lane]);
        int4 *dst = reinterpret_cast<int4 *>(nbr + nb_row(i, maxn) + nb_col(cnt & ~7));
        dst[0] = src[0];
        dst[1] = src[1];
    }
}

// Rows of every molecule of cell c (0-based extended index) of system y, by
// one warp.  Returns BUILD_OVER_* bits when a row or a bond set overflowed
// (the counts past the capacity are still reported through max_nbr).
template <bool POLY, bool TILE = false>
__device__ uint32_t build_cell(const CellSys &y, int c, BuildShared<POLY, TILE> &sh, int lane)
{
    const int ne0 = y.ne[0], ne1 = y.ne[1], ne2 = y.ne[2];
    const int cstart = y.cell_start[c] - y.mol_off;
    const int ccount = y.cell_start[c + 1] - y.mol_off - cstart;
    if (ccount == 0) return 0u;  // uniform across the warp
    const double4 *P = y.P;
    const int maxn = TILE ? y.maxn16 : y.maxn;
    const unsigned lt = (1u << lane) - 1u;
    const double csmax = fmax(y.cs[0], fmax(y.cs[1], y.cs[2]));
    const float band = (float)(1e-4 * csmax * csmax) + 1e-6f;
    const float lo32 = (float)y.rn2 - band, hi32 = (float)y.rn2 + band;
    // candidate pruning radius^2: rneighbr (1 + 5e-5) + 1e-4, far above the
    // error of the FP32 offsets (~1e-6)
    const float prune2 = (float)(y.rn2 * 1.0001 + 1e-4);
    const int cx = c % ne0, cy = (c / ne0) % ne1, cz = c / (ne0 * ne1);
    const bool chalo = is_halo(cx, ne0) || is_halo(cy, ne1) || is_halo(cz, ne2);
    if (y.dd && chalo) {  // a subdomain's halo copies are partners only: no rows
        for (int k = lane; k < ccount; k += 32) y.nnbr[cstart + k] = 0;
        return 0u;
    }
    const double refx = (cx + y.org[0] - 0.5) * y.cs[0] - y.hd[0];
    const double refy = (cy + y.org[1] - 0.5) * y.cs[1] - y.hd[1];
    const double refz = (cz + y.org[2] - 0.5) * y.cs[2] - y.hd[2];

    // --- segments of neighbour cell q = lane ---
    int n_real = 0, b_real = 0, n_img = 0, b_img = 0, code_img = NB_NOSHIFT;
    int lb_real = 0, lb_img = 0;
    if (lane < 27) {
        const int x2 = cx + lane % 3 - 1, y2 = cy + (lane / 3) % 3 - 1, z2 = cz + lane / 9 - 1;
        if (TILE && x2 >= 0 && y2 >= 0 && z2 >= 0 && x2 < ne0 && y2 < ne1 && z2 < ne2) {
            // union cell of (x2, y2, z2) around the owner's 2x2x2 block
            const int blk = tile_block_of(y.tnb, cx, cy, cz);
            const int u = (x2 - (cx & ~1) + 1) + TILE_UE * ((y2 - (cy & ~1) + 1) + TILE_UE * (z2 - (cz & ~1) + 1));
            const int32_t *bo = y.blk_off + (size_t)blk * TILE_NSEGP + 2 * u;
            lb_real = bo[0];
            lb_img = bo[1];
        }
        if (x2 >= 0 && y2 >= 0 && z2 >= 0 && x2 < ne0 && y2 < ne1 && z2 < ne2) {
            const bool h2 = is_halo(x2, ne0) || is_halo(y2, ne1) || is_halo(z2, ne2);
            if (!(chalo && h2)) {
                const int c2 = x2 + ne0 * (y2 + ne1 * z2);
                b_real = y.cell_start[c2] - y.mol_off;
                n_real = y.cell_start[c2 + 1] - y.mol_off - b_real;
                if (h2 && !y.dd) {
                    // images in a halo cell come from the interior cell on the far
                    // side: low halo <- last interior cell shifted by -domain, high
                    // halo <- first interior cell shifted by +domain
                    const int ssx = x2 == 0 ? -1 : (x2 == ne0 - 1 ? 1 : 0);
                    const int ssy = y2 == 0 ? -1 : (y2 == ne1 - 1 ? 1 : 0);
                    const int ssz = z2 == 0 ? -1 : (z2 == ne2 - 1 ? 1 : 0);
                    const int xs = x2 == 0 ? ne0 - 2 : (x2 == ne0 - 1 ? 1 : x2);
                    const int ys = y2 == 0 ? ne1 - 2 : (y2 == ne1 - 1 ? 1 : y2);
                    const int zs = z2 == 0 ? ne2 - 2 : (z2 == ne2 - 1 ? 1 : z2);
                    const int cs2 = xs + ne0 * (ys + ne1 * zs);
                    b_img = y.cell_start[cs2] - y.mol_off;
                    n_img = y.cell_start[cs2 + 1] - y.mol_off - b_img;
                    code_img = (ssx + 1) | ((ssy + 1) << 2) | ((ssz + 1) << 4);
                }
            }
        }
    }
    const int tot = n_real + n_img;
    int incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    const int excl = incl - tot;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();
    if (lane < 27) {
        sh.off[2 * lane] = excl;
        sh.off[2 * lane + 1] = excl + n_real;
        sh.start[2 * lane] = b_real;
        sh.start[2 * lane + 1] = b_img;
        sh.code[2 * lane] = NB_NOSHIFT;
        sh.code[2 * lane + 1] = code_img;
        if (TILE) {
            sh.lbase[2 * lane] = lb_real;
            sh.lbase[2 * lane + 1] = lb_img;
        }
    }
    if (lane == 0) sh.off[54] = total;
    __syncwarp();

    uint32_t over = 0u;
    for (int pass = 0; pass * 32 < ccount; pass++) {
        const int mine = pass * 32 + lane;
        const bool own = mine < ccount;
        const int i = cstart + (own ? mine : 0);
        const double4 pi = ldg_pos(P + i);
        const float xif = (float)(pi.x - refx), yif = (float)(pi.y - refy), zif = (float)(pi.z - refz);
        // bounding box of this pass's owners (lanes without an owner repeat owner 0)
        const float bx0 = warp_min(xif), bx1 = warp_max(xif);
        const float by0 = warp_min(yif), by1 = warp_max(yif);
        const float bz0 = warp_min(zif), bz1 = warp_max(zif);
        int cnt = 0, nb = 0;  // the owner lane's list and bond counts
        uint16_t *const row16 = TILE ? y.nbr16 + tile_row16(i, maxn) : nullptr;
        const int self_e = i | (NB_NOSHIFT << NB_SHIFT_BITS);  // the owner's own entry
        const int nown = min(32, ccount - pass * 32);
        __syncwarp();
        sh.ox[lane] = own ? xif : 1e30f;  // far sentinels: r^2 = inf, never a hit
        sh.oy[lane] = own ? yif : 1e30f;
        sh.oz[lane] = own ? zif : 1e30f;
        sh.oi[lane] = i;
        if (POLY) {
            sh.ochain[lane] = own ? y.chain[i] : -1;
            sh.obf[lane] = own ? y.bflag[i] : make_int4(0, 0, 0, 0);
        }
        for (int base = 0; base < total; base += NB_STAGE) {
            const int take = min(NB_STAGE, total - base);
            __syncwarp();
            // stage the window's candidates that can lie within rneighbr of
            // some owner of this pass, in visiting order (ballot compaction)
            int kept = 0;
            for (int t0 = 0; t0 < take; t0 += 32) {
                const int t = t0 + lane;
                bool keep = false;
                float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
                int j = 0, loc = 0;
                if (t < take) {
                    const int q = base + t;
                    int k = 0;  // segment containing q: largest k with off[k] <= q
#pragma unroll
                    for (int step = 32; step > 0; step >>= 1)
                        if (k + step < 54 && sh.off[k + step] <= q) k += step;
                    j = sh.start[k] + (q - sh.off[k]);
                    if (TILE) loc = tile_boff(sh.lbase[k] + (q - sh.off[k]), y.tR);
                    const int code = sh.code[k];
                    const double4 pj = ldg_pos(P + j);
                    const double xj = image(pj.x, (code & 3) - 1, y.L[0]);
                    const double yj = image(pj.y, ((code >> 2) & 3) - 1, y.L[1]);
                    const double zj = image(pj.z, ((code >> 4) & 3) - 1, y.L[2]);
                    f = make_float4((float)(xj - refx), (float)(yj - refy), (float)(zj - refz),
                                    __int_as_float(j | (code << NB_SHIFT_BITS)));
                    // squared distance from the owners' box: beyond prune2 no
                    // owner of this pass can be within rneighbr
                    const float ex = fmaxf(fmaxf(bx0 - f.x, f.x - bx1), 0.f);
                    const float ey = fmaxf(fmaxf(by0 - f.y, f.y - by1), 0.f);
                    const float ez = fmaxf(fmaxf(bz0 - f.z, f.z - bz1), 0.f);
                    keep = POLY || ex * ex + ey * ey + ez * ez < prune2;
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int pos = kept + __popc(m & lt);
                    sh.f[pos] = f;
                    if (TILE) sh.loc[pos] = (unsigned short)loc;
                    if (POLY) sh.cs[pos] = make_int2(y.chain[j], y.subchain[j]);
                }
                kept += __popc(m);
            }
            __syncwarp();
            // lane = candidate, loop over owners
            for (int t0 = 0; t0 < kept; t0 += 32) {
                const int cq = t0 + lane;
                const bool valid = cq < kept;
                // candidate sentinel on the other side: r^2 = inf against every owner
                const float4 f = valid ? sh.f[cq] : make_float4(-1e30f, -1e30f, -1e30f, 0.f);
                const int e = __float_as_int(f.w);
                const unsigned long long fx2 = pack_f32x2(f.x, f.x), fy2 = pack_f32x2(f.y, f.y),
                                         fz2 = pack_f32x2(f.z, f.z);
                int2 cs = make_int2(-2, 0);
                if (POLY && valid) cs = sh.cs[cq];
                unsigned mine_reg = 0u;  // polymers: the owner lane keeps its ballot in a register
                // owners in groups of NB_OG (pairs in packed FP32): independent chains
                // for the scheduler
                for (int o0 = 0; o0 < nown; o0 += NB_OG) {
                    bool hit[NB_OG], exact[NB_OG];
                    float r2f[NB_OG];
                    bool anyx = false;
#pragma unroll
                    for (int h = 0; h < NB_OG; h += 2) {
                        const unsigned long long dx = sub_f32x2(lds_f32x2(&sh.ox[o0 + h]), fx2);
                        const unsigned long long dy = sub_f32x2(lds_f32x2(&sh.oy[o0 + h]), fy2);
                        const unsigned long long dz = sub_f32x2(lds_f32x2(&sh.oz[o0 + h]), fz2);
                        const unsigned long long t = fma_f32x2(dz, dz, fma_f32x2(dy, dy, mul_f32x2(dx, dx)));
                        r2f[h] = __uint_as_float((unsigned)t);
                        r2f[h + 1] = __uint_as_float((unsigned)(t >> 32));
                    }
#pragma unroll
                    for (int u = 0; u < NB_OG; u++) {
                        // the band around rneighbr2 is decided in FP64; the owner
                        // itself (r2f exactly 0) is a hit here, dropped at the append
                        hit[u] = r2f[u] < lo32 && (!POLY || r2f[u] > 0.f);
                        exact[u] = !hit[u] && r2f[u] <= hi32;
                        anyx |= exact[u];
                    }
                    if (__any_sync(0xffffffffu, anyx)) {
#pragma unroll
                        for (int u = 0; u < NB_OG; u++)
                            if (exact[u]) hit[u] = exact_pair(P, sh.oi[o0 + u], e, y.L, y.rn2);
                    }
#pragma unroll
                    for (int u = 0; u < NB_OG; u++) {
                        const unsigned m = __ballot_sync(0xffffffffu, hit[u]);
                        if (POLY) {
                            if (lane == o0 + u) mine_reg = m;
                        } else if (lane == 0) {
                            sh.hits[o0 + u] = m;
                        }
                    }
                    if (POLY) {
                        int addb = 0;
#pragma unroll
                        for (int u = 0; u < NB_OG; u++) {
                            bool bond = false;
                            if (valid && o0 + u < nown && cs.x == sh.ochain[o0 + u] &&
                                !((e & NB_INDEX_MASK) == sh.oi[o0 + u] && (e >> NB_SHIFT_BITS) == NB_NOSHIFT)) {
                                const int pos = cs.y - 1, grp = pos / 31, ex = pos % 31;
                                const int4 bf = sh.obf[o0 + u];
                                const int word = grp == 0 ? bf.x : grp == 1 ? bf.y : grp == 2 ? bf.z : bf.w;
                                bond = pos >= 0 && grp < 4 && ((word >> ex) & 1);
                            }
                            const unsigned mb = __ballot_sync(0xffffffffu, bond);
                            const int b0 = __shfl_sync(0xffffffffu, nb, o0 + u);
                            if (bond) {
                                const int k = b0 + __popc(mb & lt);
                                if (k < 4) y.bnd[(size_t)sh.oi[o0 + u] * 4 + k] = e;
                            }
                            if (lane == o0 + u) addb = __popc(mb);
                        }
                        nb += addb;
                    }
                }
                // the owner lane appends its hits in candidate order, all but
                // itself, through its chunk buffer (whole sectors to the row)
                if (!POLY) __syncwarp();
                unsigned mine_hits = POLY ? mine_reg : (lane < nown ? sh.hits[lane] : 0u);
                while (mine_hits) {
                    const int b = __ffs(mine_hits) - 1;
                    mine_hits &= mine_hits - 1u;
                    const int ent = __float_as_int(sh.f[t0 + b].w);
                    if (POLY || ent != self_e) {
                        if (cnt < maxn) append_entry<TILE>(sh, lane, y.tT, y.nbr, row16, i, maxn, cnt, ent,
                                                           TILE ? sh.loc[t0 + b] : (unsigned short)0);
                        cnt++;
                    }
                }
                if (!POLY) __syncwarp();
            }
        }
        if (own && cnt < maxn) flush_entries<TILE>(sh, lane, y.tT, y.nbr, row16, i, maxn, cnt, y.tdummy);
        if (own) {
            y.nnbr[i] = cnt < maxn ? cnt : maxn;
            atomicMax(y.max_nbr, cnt);
            if (cnt > maxn) over |= BUILD_OVER_LIST;
            if (POLY) {
                y.nbond[i] = nb < 4 ? nb : 4;
                if (nb > 4) over |= BUILD_OVER_BONDS;  // too_many_bonds_error
            }
        }
    }
    __syncwarp();
    return over;
}

// ---------------------------------------------------------------------------
// Sparse systems (few molecules per cell, e.g. WCA or FENE at r_n ~ 1.4-1.5):
// one warp per block of 2x2x2 cells.  The candidates of the union of the
// owners' neighbourhoods (4x4x4 cells, each real then images, in (z, y, x)
// cell order) are staged once; each owner accepts only the candidates of its
// own 27 cells (not both halo), so its row is exactly build_cell's row, in the
// same order (the owner's cells are a sub-box of the union, visited in the same
// lexicographic order).
// ---------------------------------------------------------------------------

constexpr int NB_BSEG = 128;  // 64 union cells x (real, images)

template <bool POLY, bool TILE = false>
struct BlockShared {
    float4 f[NB_STAGE];             // candidate offsets from the block centre, entry bits in w
    alignas(16) float ox[32];       // owners (+1e30 past the last owner)
    alignas(16) float oy[32];
    alignas(16) float oz[32];
    int oi[32];
    unsigned oallow[32];            // one-hot bit of the owner's cell in the block, 0 past the last
    unsigned char allow[NB_STAGE];  // owner cells a staged candidate may pair with
    int2 cs[POLY ? NB_STAGE : 1];
    int off[NB_BSEG + 1];
    int start[NB_BSEG], code[NB_BSEG];
    int lbase[TILE ? NB_BSEG : 1];               // segment k's first candidate in the block staging
    unsigned short loc[TILE ? NB_STAGE : 1];     // staged candidates' staging offsets
    alignas(16) int ob[TILE ? 1 : 32][8];        // owner lane's chunk being filled (generic rows)
    alignas(16) unsigned short ob16[TILE ? 32 : 1][32];  // (tiled rows, 4 T <= 32 entries)
    unsigned char segallow[NB_BSEG];
    int opre[9], ostart[8];         // owners by block cell: prefix counts, first molecule
    int ochain[POLY ? 32 : 1];
    alignas(16) int4 obf[POLY ? 32 : 1];
    unsigned hits[POLY ? 1 : 32];   // per owner: which of the 32 candidates hit (polymers: registers)
};

template <bool POLY, bool TILE = false>
__device__ uint32_t build_block(const CellSys &y, int blk, BlockShared<POLY, TILE> &sh, int lane)
{
    const int ne0 = y.ne[0], ne1 = y.ne[1], ne2 = y.ne[2];
    const int nb0 = (ne0 + 1) / 2, nb1 = (ne1 + 1) / 2;
    const int bx0 = 2 * (blk % nb0), by0 = 2 * ((blk / nb0) % nb1), bz0 = 2 * (blk / (nb0 * nb1));
    const unsigned lt = (1u << lane) - 1u;
    const double4 *P = y.P;
    const int maxn = TILE ? y.maxn16 : y.maxn;

    // --- the block's owner cells (lanes 0..7: a + 2b + 4c) ---
    int ocount = 0, ostart = 0;
    bool ohalo = false;
    if (lane < 8) {
        const int x = bx0 + (lane & 1), yy = by0 + ((lane >> 1) & 1), z = bz0 + (lane >> 2);
        if (x < ne0 && yy < ne1 && z < ne2) {
            const int c = x + ne0 * (yy + ne1 * z);
            ostart = y.cell_start[c] - y.mol_off;
            ocount = y.cell_start[c + 1] - y.mol_off - ostart;
            ohalo = is_halo(x, ne0) || is_halo(yy, ne1) || is_halo(z, ne2);
            if (y.dd && ohalo) {  // a subdomain's halo copies: no rows
                for (int k = 0; k < ocount; k++) y.nnbr[ostart + k] = 0;
                ocount = 0;
            }
        }
    }
    int oincl = ocount;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, oincl, o);
        if (lane >= o) oincl += t;
    }
    const int nowners = __shfl_sync(0xffffffffu, oincl, 7);
    if (nowners == 0) return 0u;  // uniform across the warp
    const unsigned ohalo_bits = __ballot_sync(0xffffffffu, lane < 8 && ohalo) & 0xffu;
    __syncwarp();
    if (lane < 8) { sh.opre[lane + 1] = oincl; sh.ostart[lane] = ostart; }
    if (lane == 0) sh.opre[0] = 0;

    const double csmax = fmax(y.cs[0], fmax(y.cs[1], y.cs[2]));
    const float band = (float)(1e-4 * csmax * csmax) + 1e-6f;
    const float lo32 = (float)y.rn2 - band, hi32 = (float)y.rn2 + band;
    const float prune2 = (float)(y.rn2 * 1.0001 + 1e-4);
    const double refx = (bx0 + y.org[0]) * y.cs[0] - y.hd[0];  // centre of the 2x2x2 block
    const double refy = (by0 + y.org[1]) * y.cs[1] - y.hd[1];
    const double refz = (bz0 + y.org[2]) * y.cs[2] - y.hd[2];

    // --- segments of the union cells u = lane and u = lane + 32 ---
    int seg_n[4], seg_b[4], seg_code[4];
    unsigned seg_allow[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int u = lane + 32 * h;
        const int ux = u & 3, uy = (u >> 2) & 3, uz = u >> 4;
        const int x2 = bx0 - 1 + ux, y2 = by0 - 1 + uy, z2 = bz0 - 1 + uz;
        seg_n[2 * h] = seg_n[2 * h + 1] = 0;
        seg_b[2 * h] = seg_b[2 * h + 1] = 0;
        seg_code[2 * h] = seg_code[2 * h + 1] = NB_NOSHIFT;
        seg_allow[h] = 0u;
        if (x2 >= 0 && y2 >= 0 && z2 >= 0 && x2 < ne0 && y2 < ne1 && z2 < ne2) {
            const bool h2 = is_halo(x2, ne0) || is_halo(y2, ne1) || is_halo(z2, ne2);
            // owner cells (a, b, c) whose 27 neighbours include u, not both halo
            unsigned al = 0u;
#pragma unroll
            for (int oc = 0; oc < 8; oc++) {
                const int a = oc & 1, b = (oc >> 1) & 1, cc = oc >> 2;
                const bool adj = ux >= a && ux <= a + 2 && uy >= b && uy <= b + 2 && uz >= cc && uz <= cc + 2;
                if (adj && !(h2 && ((ohalo_bits >> oc) & 1u))) al |= 1u << oc;
            }
            seg_allow[h] = al;
            if (al) {
                const int c2 = x2 + ne0 * (y2 + ne1 * z2);
                seg_b[2 * h] = y.cell_start[c2] - y.mol_off;
                seg_n[2 * h] = y.cell_start[c2 + 1] - y.mol_off - seg_b[2 * h];
                if (h2 && !y.dd) {
                    // images of the interior cell on the far side, as in build_cell
                    const int ssx = x2 == 0 ? -1 : (x2 == ne0 - 1 ? 1 : 0);
                    const int ssy = y2 == 0 ? -1 : (y2 == ne1 - 1 ? 1 : 0);
                    const int ssz = z2 == 0 ? -1 : (z2 == ne2 - 1 ? 1 : 0);
                    const int xs = x2 == 0 ? ne0 - 2 : (x2 == ne0 - 1 ? 1 : x2);
                    const int ys = y2 == 0 ? ne1 - 2 : (y2 == ne1 - 1 ? 1 : y2);
                    const int zs = z2 == 0 ? ne2 - 2 : (z2 == ne2 - 1 ? 1 : z2);
                    const int cs2 = xs + ne0 * (ys + ne1 * zs);
                    seg_b[2 * h + 1] = y.cell_start[cs2] - y.mol_off;
                    seg_n[2 * h + 1] = y.cell_start[cs2 + 1] - y.mol_off - seg_b[2 * h + 1];
                    seg_code[2 * h + 1] = (ssx + 1) | ((ssy + 1) << 2) | ((ssz + 1) << 4);
                }
            }
        }
    }
    // prefix over the 128 segments in union-cell order: cells 0..31, then 32..63
    int carry = 0;
    __syncwarp();
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int tot = seg_n[2 * h] + seg_n[2 * h + 1];
        int incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int excl = carry + incl - tot;
        const int u = lane + 32 * h;
        sh.off[2 * u] = excl;
        sh.off[2 * u + 1] = excl + seg_n[2 * h];
        sh.start[2 * u] = seg_b[2 * h];
        sh.start[2 * u + 1] = seg_b[2 * h + 1];
        sh.code[2 * u] = seg_code[2 * h];
        sh.code[2 * u + 1] = seg_code[2 * h + 1];
        sh.segallow[2 * u] = (unsigned char)seg_allow[h];
        sh.segallow[2 * u + 1] = (unsigned char)seg_allow[h];
        if (TILE) {  // the same block and segments as the tiled force staging
            const int32_t *bo = y.blk_off + (size_t)blk * TILE_NSEGP + 2 * u;
            sh.lbase[2 * u] = bo[0];
            sh.lbase[2 * u + 1] = bo[1];
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    const int total = carry;
    if (lane == 0) sh.off[NB_BSEG] = total;
    __syncwarp();

    uint32_t over = 0u;
    for (int pass = 0; pass * 32 < nowners; pass++) {
        const int k = pass * 32 + lane;
        const bool own = k < nowners;
        const int kk = own ? k : 0;  // lanes without an owner read owner 0
        int oc = 0;                  // the owner's block cell: the last oc with opre[oc] <= kk
#pragma unroll
        for (int q = 1; q < 8; q++) oc += kk >= sh.opre[q] ? 1 : 0;
        const int i = sh.ostart[oc] + (kk - sh.opre[oc]);
        const double4 pi = ldg_pos(P + i);
        const float xif = (float)(pi.x - refx), yif = (float)(pi.y - refy), zif = (float)(pi.z - refz);
        const float bx_lo = warp_min(own ? xif : 3e38f), bx_hi = warp_max(own ? xif : -3e38f);
        const float by_lo = warp_min(own ? yif : 3e38f), by_hi = warp_max(own ? yif : -3e38f);
        const float bz_lo = warp_min(own ? zif : 3e38f), bz_hi = warp_max(own ? zif : -3e38f);
        int cnt = 0, nb = 0;
        uint16_t *const row16 = TILE ? y.nbr16 + tile_row16(i, maxn) : nullptr;
        const int self_e = i | (NB_NOSHIFT << NB_SHIFT_BITS);  // the owner's own entry
        const int nown = min(32, nowners - pass * 32);
        __syncwarp();
        sh.ox[lane] = own ? xif : 1e30f;
        sh.oy[lane] = own ? yif : 1e30f;
        sh.oz[lane] = own ? zif : 1e30f;
        sh.oi[lane] = i;
        sh.oallow[lane] = own ? 1u << oc : 0u;
        if (POLY) {
            sh.ochain[lane] = own ? y.chain[i] : -1;
            sh.obf[lane] = own ? y.bflag[i] : make_int4(0, 0, 0, 0);
        }
        for (int base = 0; base < total; base += NB_STAGE) {
            const int take = min(NB_STAGE, total - base);
            __syncwarp();
            int kept = 0;
            for (int t0 = 0; t0 < take; t0 += 32) {
                const int t = t0 + lane;
                bool keep = false;
                float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
                unsigned al = 0u;
                int j = 0, loc = 0;
                if (t < take) {
                    const int q = base + t;
                    int kk = 0;  // segment containing q: largest kk with off[kk] <= q
#pragma unroll
                    for (int step = 64; step > 0; step >>= 1)
                        if (kk + step < NB_BSEG && sh.off[kk + step] <= q) kk += step;
                    j = sh.start[kk] + (q - sh.off[kk]);
                    if (TILE) loc = tile_boff(sh.lbase[kk] + (q - sh.off[kk]), y.tR);
                    const int code = sh.code[kk];
                    al = sh.segallow[kk];
                    const double4 pj = ldg_pos(P + j);
                    const double xj = image(pj.x, (code & 3) - 1, y.L[0]);
                    const double yj = image(pj.y, ((code >> 2) & 3) - 1, y.L[1]);
                    const double zj = image(pj.z, ((code >> 4) & 3) - 1, y.L[2]);
                    f = make_float4((float)(xj - refx), (float)(yj - refy), (float)(zj - refz),
                                    __int_as_float(j | (code << NB_SHIFT_BITS)));
                    const float ex = fmaxf(fmaxf(bx_lo - f.x, f.x - bx_hi), 0.f);
                    const float ey = fmaxf(fmaxf(by_lo - f.y, f.y - by_hi), 0.f);
                    const float ez = fmaxf(fmaxf(bz_lo - f.z, f.z - bz_hi), 0.f);
                    keep = POLY || ex * ex + ey * ey + ez * ez < prune2;
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int pos = kept + __popc(m & lt);
                    sh.f[pos] = f;
                    sh.allow[pos] = (unsigned char)al;
                    if (TILE) sh.loc[pos] = (unsigned short)loc;
                    if (POLY) sh.cs[pos] = make_int2(y.chain[j], y.subchain[j]);
                }
                kept += __popc(m);
            }
            __syncwarp();
            for (int t0 = 0; t0 < kept; t0 += 32) {
                const int cq = t0 + lane;
                const bool valid = cq < kept;
                const float4 f = valid ? sh.f[cq] : make_float4(-1e30f, -1e30f, -1e30f, 0.f);
                const unsigned callow = valid ? sh.allow[cq] : 0u;
                const int e = __float_as_int(f.w);
                const unsigned long long fx2 = pack_f32x2(f.x, f.x), fy2 = pack_f32x2(f.y, f.y),
                                         fz2 = pack_f32x2(f.z, f.z);
                int2 cs = make_int2(-2, 0);
                if (POLY && valid) cs = sh.cs[cq];
                unsigned mine_reg = 0u;  // polymers: the owner lane keeps its ballot in a register
                for (int o0 = 0; o0 < nown; o0 += NB_OG) {
                    bool hit[NB_OG], exact[NB_OG];
                    float r2f[NB_OG];
                    bool anyx = false;
#pragma unroll
                    for (int h = 0; h < NB_OG; h += 2) {
                        const unsigned long long dx = sub_f32x2(lds_f32x2(&sh.ox[o0 + h]), fx2);
                        const unsigned long long dy = sub_f32x2(lds_f32x2(&sh.oy[o0 + h]), fy2);
                        const unsigned long long dz = sub_f32x2(lds_f32x2(&sh.oz[o0 + h]), fz2);
                        const unsigned long long t = fma_f32x2(dz, dz, fma_f32x2(dy, dy, mul_f32x2(dx, dx)));
                        r2f[h] = __uint_as_float((unsigned)t);
                        r2f[h + 1] = __uint_as_float((unsigned)(t >> 32));
                    }
#pragma unroll
                    for (int u = 0; u < NB_OG; u++) {
                        const bool ok = (callow & sh.oallow[o0 + u]) != 0u;
                        // the owner itself: dropped at the append (polymers: decided in FP64)
                        hit[u] = ok && r2f[u] < lo32 && (!POLY || r2f[u] > 0.f);
                        exact[u] = ok && !hit[u] && r2f[u] <= hi32;
                        anyx |= exact[u];
                    }
                    if (__any_sync(0xffffffffu, anyx)) {
#pragma unroll
                        for (int u = 0; u < NB_OG; u++)
                            if (exact[u]) hit[u] = exact_pair(P, sh.oi[o0 + u], e, y.L, y.rn2);
                    }
#pragma unroll
                    for (int u = 0; u < NB_OG; u++) {
                        const unsigned m = __ballot_sync(0xffffffffu, hit[u]);
                        if (POLY) {
                            if (lane == o0 + u) mine_reg = m;
                        } else if (lane == 0) {
                            sh.hits[o0 + u] = m;
                        }
                    }
                    if (POLY) {
                        int addb = 0;
#pragma unroll
                        for (int u = 0; u < NB_OG; u++) {
                            bool bond = false;
                            if ((callow & sh.oallow[o0 + u]) != 0u && cs.x == sh.ochain[o0 + u] &&
                                !((e & NB_INDEX_MASK) == sh.oi[o0 + u] && (e >> NB_SHIFT_BITS) == NB_NOSHIFT)) {
                                const int pos = cs.y - 1, grp = pos / 31, ex = pos % 31;
                                const int4 bf = sh.obf[o0 + u];
                                const int word = grp == 0 ? bf.x : grp == 1 ? bf.y : grp == 2 ? bf.z : bf.w;
                                bond = pos >= 0 && grp < 4 && ((word >> ex) & 1);
                            }
                            const unsigned mb = __ballot_sync(0xffffffffu, bond);
                            const int b0 = __shfl_sync(0xffffffffu, nb, o0 + u);
                            if (bond) {
                                const int kb = b0 + __popc(mb & lt);
                                if (kb < 4) y.bnd[(size_t)sh.oi[o0 + u] * 4 + kb] = e;
                            }
                            if (lane == o0 + u) addb = __popc(mb);
                        }
                        nb += addb;
                    }
                }
                // the owner lane appends its hits in candidate order, all but
                // itself, through its chunk buffer (whole sectors to the row)
                if (!POLY) __syncwarp();
                unsigned mine_hits = POLY ? mine_reg : (lane < nown ? sh.hits[lane] : 0u);
                while (mine_hits) {
                    const int b = __ffs(mine_hits) - 1;
                    mine_hits &= mine_hits - 1u;
                    const int ent = __float_as_int(sh.f[t0 + b].w);
                    if (POLY || ent != self_e) {
                        if (cnt < maxn) append_entry<TILE>(sh, lane, y.tT, y.nbr, row16, i, maxn, cnt, ent,
                                                           TILE ? sh.loc[t0 + b] : (unsigned short)0);
                        cnt++;
                    }
                }
                if (!POLY) __syncwarp();
            }
        }
        if (own && cnt < maxn) flush_entries<TILE>(sh, lane, y.tT, y.nbr, row16, i, maxn, cnt, y.tdummy);
        if (own) {
            y.nnbr[i] = cnt < maxn ? cnt : maxn;
            atomicMax(y.max_nbr, cnt);
            if (cnt > maxn) over |= BUILD_OVER_LIST;
            if (POLY) {
                y.nbond[i] = nb < 4 ? nb : 4;
                if (nb > 4) over |= BUILD_OVER_BONDS;
            }
        }
    }
    __syncwarp();
    return over;
}

}  // namespace fm
