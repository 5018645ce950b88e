// fm_common.cuh -- device data layout and kernel launch interface of the
// B200 MD hot path (single system).  Host code (fm_api.cu) owns an FmSystem;
// kernels (fm_kernels.cu) receive an FmDev by value.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fm {

// ---- status word bits (FmScalars::status) -------------------------------
// A set FATAL bit freezes the step loop: every later kernel returns at entry,
// so the device state stays exactly as it was when the fault was detected.
enum : uint32_t {
    ST_ESCAPE = 1u << 0,    // molecule binned outside the extended cell grid
    ST_NLIST = 1u << 1,     // a neighbour list needed more than maxn slots
    ST_PE = 1u << 2,        // per-molecule PE above 10000 on a record step
    ST_BOND = 1u << 3,      // FENE bond at or beyond R_0
    ST_TILE = 1u << 4,      // a block's staged neighbourhood exceeded the tiled force kernel's capacity
    ST_ANGLE = 1u << 5,     // angular triple with no defined result (missing bond, k_ijk < 1e-5)
    ST_MIGRATE = 1u << 6,   // subdomain: a molecule left the neighbouring subdomains, or the capacity ran out
    ST_FATAL = ST_ESCAPE | ST_NLIST | ST_PE | ST_BOND | ST_TILE | ST_ANGLE | ST_MIGRATE,
};

// Device-resident scalars of the step loop (one per system).
struct FmScalars {
    double rmax;              // simulation_checkrebuild.f90 `rmax` (save variable)
    unsigned long long vmax2; // bits of max |v|^2 (non-negative doubles order like u64)
    int32_t rebuild;          // decision for the current iteration
    int32_t pset;             // which position buffer is current
    uint32_t status;          // ST_* bits
    int32_t fail_iter;        // iteration at which a FATAL bit was first set
    int32_t max_nbr;          // largest neighbour count seen at the last build
    int32_t escape_slot;      // a molecule that escaped (internal slot)
    int64_t rebuilds;         // rebuilds performed
    uint64_t digest;          // pair-set digest (test hook)
    int64_t digest_n;
    int32_t nrec_pending;     // record rows written since the host last read
    int32_t build_next;       // list build: next work unit to hand out (zeroed before each build)
    int32_t disp_reset;       // rebuild criterion 2: the last decision rebuilt, so rdisp restarts at 0
    unsigned long long dmax;  // rebuild criterion 2: bits of max |rdisp component| this step
    double pacc[6];           // pressure_outflag 1: sum over samples of P (xx yy zz xy xz yz)
    int32_t pcount;           // samples in pacc
    int32_t tile_next;        // tiled force kernel: next block to hand out (the last taker resets it)
    int32_t umax;             // tiled path: largest staged neighbourhood seen at the last build
    int32_t g_iter;           // rebuild graph: iteration its next decision is for
    int32_t cur_iter;         // rebuild graph: iteration of the last decision (errors in its body)
    int64_t graph_kernels;    // rebuild graph: kernels its conditional body has run
};

// Iteration argument of a kernel inside the rebuild graph's body: the
// iteration of the decision that opened the body (FmScalars::cur_iter).
constexpr int ITER_DEVICE = -2147483647 - 1;

// Partial sums of one record step, one row per force-kernel block.
// With pressure_outflag 1 the six distinct components of v v + rf/2 follow
// (cumulative_pressure case 1, simulation_record.f90:3151-3220).
enum { RS_PE = 0, RS_VIR, RS_MV2, RS_VSUM, RS_PEMAX, RS_PXX, RS_PYY, RS_PZZ, RS_PXY, RS_PXZ, RS_PYZ, RS_N };

// Record row layout in device memory (matches fm_macro on the host).
struct FmRecord {
    int32_t iter;
    int32_t pad_;
    double simtime, vsum, mv2sum, temperature, kinenergy, potenergy, totenergy, pressure, virial;
};

// Everything a kernel needs, passed by value.
// Mie pair constants for one (type_i, type_j), precombined in the
// reference's evaluation order: Mie_accijmag = (C eps)(lr s^(lr/2+1) -
// (alpha la) s^(la/2+1)), Mie_energy = (C eps)(s^(lr/2) - alpha s^(la/2)) -
// potshift, harmonic bonds -k (r - r0)/r and k/2 (r - r0)^2.
constexpr int MIE_MAXT = 16;

// Soddemann solvent (polymer_info_MD, modules.f90:456-462).  sod_a, sod_b and
// wca_cut2 are written there as default-real literals, so the FP64 parameters
// hold their single-precision roundings: these are those values, exactly.
constexpr double SOD_CUT = 1.5, SOD_CUT2 = 2.25;
constexpr double SOD_A = 0x1.96274p+1;         // 3.1730728678 as REAL(4) = 3.1730728149414062
constexpr double SOD_B = -0x1.b6639ap-1;       // -0.85622864544 as REAL(4) = -0.8562286496162415
constexpr double SOD_WCA_CUT2 = 0x1.428a3p+0;  // 1.25992104989487 as REAL(4) = 1.2599210739135742
struct FmMiePair {
    double ceps, lr, ala, er1, ea1, er, ea, alpha, shift, k, r0;
};

struct FmDev {
    // geometry and constants
    int n;                 // real molecules
    double L[3], hd[3], cs[3];
    int nc[3];             // interior cells per axis
    int ne[3];             // extended cells per axis (nc + 2)
    int ncell;             // ne[0]*ne[1]*ne[2]
    double rc2, rn2, dt, potshift, half_dt, half_dt2;
    double density, pot_slrc, p_slrc;
    int tplot;
    int integrator;        // 0 leap-frog, 1 velocity Verlet
    int maxn;              // neighbour slots per molecule
    int precision;
    // positions (double-buffered: pos[sc->pset] is current)
    double4 *pos0, *pos1;
    // velocities, accelerations (SoA)
    double *vx, *vy, *vz, *ax, *ay, *az;
    int32_t *slot_of;      // internal slot -> upload index (the molecule's identity)
    // reorder scratch
    double *tvx, *tvy, *tvz, *tax, *tay, *taz;
    // cells (extended grid, x fastest)
    int32_t *cell_of;      // per molecule (old order) cell id
    int32_t *cell_count;   // ncell
    int32_t *cell_start;   // ncell + 1
    int32_t *perm;         // new slot -> old slot
    int32_t *tile_sum;     // per scan tile (4096 cells)
    // neighbour list: entry k of molecule i, at nb_row(i, maxn) + nb_col(k), is
    // j | (sx+1)<<26 | (sy+1)<<28 | (sz+1)<<30
    int32_t *nbr;
    int32_t *nnbr;
    // per-molecule PE / virial (record steps)
    double *pe, *vir;
    // FENE polymers (potential_flag 1): monomer data per slot and bonds found
    // at list build, bnd[i*4 + b] = partner | image code, like nbr entries
    int potential_flag;
    double k_c, R0, R0_2;
    int32_t *chain, *subchain;
    int4 *bflag;
    int32_t *tchain, *tsubchain;
    int4 *tbflag;
    int32_t *bnd, *nbond;
    // Mie_potential 1: per-type-pair constants, per-type masses; a molecule's
    // type (1-based) rides in the w component of its position
    int build_blocks;            // list build: one warp per 2x2x2 cells (sparse systems)
    // Tiled force path (tile = 1): the extended cell grid is cut into blocks of
    // 2x2x2 cells; the force kernel stages the positions of a block's 4x4x4
    // cell neighbourhood (images applied) in shared memory, and list entries
    // are 16-bit offsets into that staging (fm_tile.cuh).
    int tile;
    int tile_T;                  // lanes per molecule (4 or 8); fixes the row layout
    int tile_R;                  // staged rows per 32 candidates: 3 (x y z) or 4 (+ w)
    int tile_nb[3];              // blocks per axis, ceil(ne / 2)
    int tile_nblk;
    int tile_ucap;               // staged candidates per block the force kernel holds
    int32_t *blk_off;            // [tile_nblk][TILE_NSEGP] prefix of the staging segments
    uint16_t *nbr16;             // rows of maxn16 entries (tile_pos16 layout)
    int maxn16;
    // pressure_outflag 1: rf (xx yy zz xy xz yz) per molecule of the last
    // record step (pressure_tensor_forces, simulation_record.f90:6239-6256)
    int pressure;
    double *rf6;
    // rebuild criterion 2: displacement since the last rebuild, per molecule
    // (simulation_checkrebuild.f90:111-121); molecules move slots only at rebuilds,
    // which restart it, so it needs no reordering
    double *rdx, *rdy, *rdz;
    // solvent_flag 1: Soddemann well depth by chain beads in the pair (eps_ss,
    // eps_ps, eps_pp); a molecule's bead flag (chainID != 0) rides in w
    int solvent;
    double sod_eps[3];
    int mie;
    // angular_potential (simulation_compute_forces_angular): k and theta_0 by
    // the Mie types of a triple, [(ti-1) + nt ((tj-1) + nt (tk-1))]; funcy by
    // slot (reordered with the chains); bonds of a middle bead (funcy 2)
    // ordered as the reference discovers them (bnd[4 j] is its i, bnd[4 j + 1]
    // its k)
    int angular, ang_nt;
    const double *ang_k, *ang_t0;
    int32_t *funcy, *tfuncy;
    const FmMiePair *mie_pair;   // [(ti-1) + MIE_MAXT*(tj-1)]
    const double *mie_mass;      // [ti-1]
    const int32_t *mie_type_up;  // moltype by upload index (written into w at upload)
    // Subdomain of a spatial decomposition (dd = 1): the extended grid above is
    // this rank's interior cells nc plus one halo layer; interior cell x = 1
    // is global interior cell org[0] (0-based) of the global grid of gne - 2
    // cells per axis, whose cell size and box (L, hd, cs) are the ones above.
    // Positions are global coordinates.  The halo cells hold explicit copies
    // of the neighbouring subdomains' boundary molecules (periodic shift
    // applied by the sender), marked by w = 1 (owned molecules: w = 0), with
    // v = a = 0 and no rows; images are never formed.
    int dd;
    int org[3], gne[3];
    // record partials [nblocks][RS_N] and finished rows
    double *partial;
    int nblocks_force;
    FmRecord *rec;
    int rec_cap;
    FmScalars *sc;
};

__host__ __device__ inline double4 *cur_pos(const FmDev &d, int pset) { return pset ? d.pos1 : d.pos0; }

// Neighbour entry encoding.
constexpr int NB_SHIFT_BITS = 26;
constexpr int32_t NB_INDEX_MASK = (1 << NB_SHIFT_BITS) - 1;
constexpr int MAX_MOLECULES = NB_INDEX_MASK;

// Neighbour list layout: molecules in groups of 32, each molecule's entries
// in chunks of 8 (one 32-byte sector); chunk c of the 32 molecules of a group
// is one contiguous 1 KB block (molecule i%32 at offset 32 (i%32) bytes), so a
// warp that reads a 16-byte half of chunk c of its 32 molecules reads 32
// sectors of one block, and the list build writes each sector whole (a
// sector shared by two molecules written at different times would reach
// DRAM half-written once the list outgrows L2).  The array holds
// ceil(n/32)*32 rows of maxn (a multiple of 8) entries.
__host__ __device__ inline size_t nb_row(int i, int maxn)
{
    return (size_t)(i >> 5) * (size_t)maxn * 32u + (size_t)(i & 31) * 8u;
}
__host__ __device__ inline size_t nb_col(int k) { return (size_t)(k & ~7) * 32u + (size_t)(k & 7); }
inline size_t nb_rows(int n) { return ((size_t)n + 31u) / 32u * 32u; }

// Subdomain bookkeeping of the decomposition kernels (fm_dd_kernels.cu).
constexpr int DD_MREC = 10;  // migrating molecule: r, v, a, global number
constexpr int DD_HREC = 5;   // halo copy: shifted r, global number, destination halo cell
struct DdDev {
    int rank, dims[3];
    const int32_t *owner_axis;  // process coordinate of each global interior cell, x then y then z
    // needs of this rank's cells: for cell c, entries [need_off[c], need_off[c+1])
    // of (rank whose halo holds it, image code it is seen with, that rank's halo cell)
    const int32_t *need_off, *need_rank, *need_code, *need_cell;
    int32_t *count, *offset, *cursor;  // per destination rank
    int32_t *nlist;                    // emigrants listed
    int32_t *list_idx, *list_aux;      // emigrant slot and destination
    int list_cap;
};
void launch_dd_classify(const FmDev &d, const DdDev &x, int n, int wrap, int iter, cudaStream_t st);
void launch_dd_pack_emigrants(const FmDev &d, const DdDev &x, int n, double *out, cudaStream_t st);
void launch_dd_append_immigrants(const FmDev &d, const DdDev &x, const double *in, int n, int base, int iter,
                                 cudaStream_t st);
void launch_dd_halo_records(const FmDev &d, const DdDev &x, int n, int pass, double *out, cudaStream_t st);
void launch_dd_append_halo(const FmDev &d, const double *in, int n, int base, cudaStream_t st);
void launch_dd_gather_positions(const FmDev &d, const int32_t *idx, const int8_t *code, int n, double *out,
                                cudaStream_t st);
void launch_dd_scatter_positions(const FmDev &d, const int32_t *idx, const double *in, int n, cudaStream_t st);
void launch_dd_sums(const FmDev &d, double *out, cudaStream_t st);

// Sets the message fm_last_error returns on this thread (fm_api.cu).
void set_last_error(const char *msg);

// ---- kernel launchers (fm_kernels.cu) -----------------------------------
// All launchers enqueue on `st` and never synchronise.
void launch_reset_scalars(const FmDev &d, cudaStream_t st);
void launch_move1(const FmDev &d, cudaStream_t st);          // pass 1 in place + vmax2
void launch_move2(const FmDev &d, cudaStream_t st);          // pass 2 in place
void launch_vmax(const FmDev &d, cudaStream_t st);           // vmax2 of current v
void launch_move_lfv(const FmDev &d, cudaStream_t st);       // leap-frog move in place + vmax2
void launch_disp(const FmDev &d, cudaStream_t st);            // criterion 2: rdisp += v dt, max component
extern thread_local bool pdl_capture;  // set while a graph is captured: launches without PDL edges
void launch_decide_graph(const FmDev &d, int flip, int rebuild_criteria, int fixed_rebuild, double half_min_delta,
                         cudaGraphConditionalHandle cond, int body_kernels, cudaStream_t st);
void launch_set_graph_iter(const FmDev &d, int iter, cudaStream_t st);
void launch_decide(const FmDev &d, int iter, int flip, int rebuild_criteria, int fixed_rebuild,
                   double half_min_delta, cudaStream_t st);
// Rebuild pipeline; gated = 1 makes each kernel a no-op unless sc->rebuild.
void launch_wrap_bin(const FmDev &d, int wrap, int bin, int gated, int iter, cudaStream_t st);
void launch_scan_cells(const FmDev &d, int gated, cudaStream_t st);
void launch_scatter(const FmDev &d, int gated, cudaStream_t st);
void launch_reorder(const FmDev &d, int gated, double4 *tpos, int32_t *tuidx, cudaStream_t st);
void launch_build_nlist(const FmDev &d, int gated, int iter, cudaStream_t st);
// angular_potential: orders each middle bead's two bonds as the reference's
// list build discovers them (after every build).
void launch_angular_order(const FmDev &d, int gated, int iter, cudaStream_t st);
void launch_set_funcy(const FmDev &d, const int32_t *funcy_up, cudaStream_t st);
// Tiled path: the staging segment table of every block (before the build).
void launch_blk_seg(const FmDev &d, int gated, int iter, cudaStream_t st);
size_t tile_smem_bytes(const FmDev &d);
int tile_ucap_limit(int R);
// Decodes the tiled rows into the generic int32 layout at `out` (rows of
// d.maxn), for the pair-list and digest test hooks.
void launch_tile_to_generic(const FmDev &d, int32_t *out, int maxn, cudaStream_t st);
// Forces: mode 0 forces only, 1 forces + move(2), 2 forces + move(2) + next
// move(1), 3 forces + leap-frog move.
void launch_force(const FmDev &d, int record, int mode, int tpm, cudaStream_t st);
void launch_record(const FmDev &d, int iter, double simtime, cudaStream_t st);
void launch_all_pairs(const FmDev &d, int record, int mode, cudaStream_t st);
// Record partials straight from the per-molecule arrays (PE, virial) and the
// current velocities, for the subroutine-by-subroutine path.
void launch_macro_partials(const FmDev &d, cudaStream_t st);
int macro_blocks(int n);
void launch_pair_digest(const FmDev &d, const int32_t *glob_of_upload, cudaStream_t st);
int force_blocks(int n, int tpm);
int scan_tiles(int ncell);
int all_pairs_blocks(int n);
// Layout conversion between the reference's (3,n) column-major arrays and
// the device layout; `order` maps upload index -> slot.
void launch_set_types(const FmDev &d, cudaStream_t st);
void launch_set_bead_flags(const FmDev &d, cudaStream_t st);
void launch_scatter_state(const FmDev &d, const double *r3, const double *v3, const double *a3,
                          cudaStream_t st);
void launch_gather_state(const FmDev &d, double *r3, double *v3, double *a3, int32_t *gid,
                         double *pe, double *vir, cudaStream_t st);

// ---- sort_mols (fm_sort.cu) ------------------------------------------------
// Device scalars of sort_mols (linklist.f90:2744-2869): its save variables
// nrebuilds (starts at 1), sf1 (1.5) and sf2 (5), and the current sort.
struct FmSortScalars {
    int32_t nrebuilds;
    int32_t due;       // this rebuild sorts
    int32_t ave;       // ave_molperblock of this sort, safety factors applied
    int32_t overflow;  // a block holds more than ave: this sort is skipped
    double sf1;
    int32_t sf2;
    int32_t pad_;
    int64_t sorts, skipped;
};
// Sort blocks of sortblocksize^3 cells, their Hcurve order and the buffers of
// the stable (block, upload index) sort.  Keys and values are by upload index.
struct FmSortDev {
    int freq, blocks, end_bit;
    int nb[3];
    double bsl[3];                // blocksidelength
    const int32_t *hc;            // Hcurve, x fastest, values 1..blocks
    int32_t *key, *key_out;       // block (0-based Hcurve value) by upload index, sorted
    int32_t *val, *val_out;       // 0..n-1, and the upload indices in sorted order
    int32_t *cnt;                 // molecules per block of the current sort
    int32_t *newv;                // new upload index of each old one
    int32_t *gtmp;                // global numbers, permuted
    int32_t *glob;                // global number by upload index (the handle's)
    void *tmp;                    // radix-sort scratch
    size_t tmp_bytes;
    FmSortScalars *ss;
};
// Hcurve for sort_flag 1 (x-fastest block numbers) or 2 (build_hilbert,
// functions_lib.f90:2555-2604) over nb blocks per axis, into out[blocks].
// Returns 0, or -1 with *why set.
int sort_table(int flag, const int nb[3], int32_t *out, const char **why);
// Radix-sort scratch bytes for n (key, value) pairs of end_bit key bits.
size_t sort_scratch_bytes(int n, int end_bit);
// The rebuild's sort_mols: counter, keys, stable sort, renumbering.  With
// `gated` the kernels run only on a rebuild step.
void launch_sort(const FmDev &d, const FmSortDev &s, int gated, cudaStream_t st);
// The same split for the rebuild graph: the counter kernel, which sets `cond`
// (a conditional node in the rebuild body) when this rebuild sorts and then
// counts body_kernels more kernels, and the node's body.
void launch_sort_gate_graph(const FmDev &d, const FmSortDev &s, cudaGraphConditionalHandle cond, int body_kernels,
                            cudaStream_t st);
void launch_sort_body(const FmDev &d, const FmSortDev &s, int gated, cudaStream_t st);

}  // namespace fm
