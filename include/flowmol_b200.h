/*
 * flowmol_b200.h -- C ABI of the B200 (sm_100a) per-timestep MD hot path.
 *
 * Every entry point replaces one Fortran subroutine (or the fused loop) of
 * Flowmol's velocity-Verlet step (md.f90:143-163, md_advance_vv).  The
 * reference subroutines take no arguments and talk through module globals;
 * here the module state lives in an opaque handle whose arrays sit in device
 * memory.  All functions return 0 on success or one of the FM_ERR_* codes; a
 * message is available from fm_last_error().  Nothing aborts the host process
 * (the reference's error_abort -> MPI_Abort, messenger.MPI.f90:3376-3410,
 * becomes a return code).  Plain C types only: callable from Fortran through
 * iso_c_binding, from Python through ctypes, from C/C++ directly.
 *
 * Threading: a handle is used by one host thread at a time; all its device
 * work is ordered on one CUDA stream (fm_set_stream).  Different handles may
 * be driven from different threads.
 */
#ifndef FLOWMOL_B200_H
#define FLOWMOL_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define FM_API __attribute__((visibility("default")))
#else
#define FM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define FM_OK 0
#define FM_ERR_ARG 1            /* invalid argument */
#define FM_ERR_CUDA 2           /* CUDA runtime failure (message has the CUDA error) */
#define FM_ERR_FEWCELLS 3       /* fewer than 3 cells per axis (setup_set_parameters.f90:1891-1896) */
#define FM_ERR_ESCAPE 4         /* molecule outside the cell grid (linklist.f90:2664-2673) */
#define FM_ERR_NLIST 5          /* neighbour list needs more capacity than the cap allows */
#define FM_ERR_PE 6             /* max per-molecule PE > 10000 (simulation_record.f90:1271-1283) */
#define FM_ERR_STATE 7          /* call made in the wrong order (e.g. step before setup) */
#define FM_ERR_BOND 8           /* polymer bond stretched beyond R_0 (setup_set_parameters.f90:352) */
#define FM_ERR_NODEVICE 9       /* no CUDA device / library not built for this GPU */
#define FM_ERR_IO 10            /* restart or input file could not be read or written */

/* ---- enumerations mirroring the reference's input flags ------------- */
#define FM_FORCE_LIST_ALLPAIRS 0   /* FORCE_LIST 0: LJ all pairs, minimum image */
#define FM_FORCE_LIST_FULL 2       /* FORCE_LIST 2: full neighbour list */
#define FM_FORCE_LIST_HALF 3       /* FORCE_LIST 3: half (Newton-3) list, the reference default */
#define FM_PRECISION_FP64 0        /* plain FP64 drop-in */
#define FM_PRECISION_FP32 1        /* FP32 pair forces, FP64 r/v/a, FP64 compensated sums */

/*
 * Parameters of one simulation (the hot-path subset of the reference's
 * input keywords, setup_read_input.f90).  Derived quantities -- halfdomain,
 * rneighbr2, ncells, cellsidelength, potshift, long-range corrections -- are
 * computed by the library with the reference's formulas
 * (setup_set_parameters.f90:1099-1245, 1848-1903).
 */
typedef struct fm_params {
    int32_t np;                   /* molecules (globalnp on one rank) */
    double domain[3];             /* box lengths (globaldomain) */
    double density;               /* DENSITY: used in pressure and sLRC */
    double rcutoff;               /* RCUTOFF */
    double delta_rneighbr[3];     /* DELTA_RNEIGHBR (skin per axis) */
    double delta_t;               /* DELTA_T */
    int32_t tplot;                /* TPLOT: record / forced-rebuild period */
    int32_t initialstep;          /* iteration number of the uploaded state */
    double simtime;               /* simulated time of the uploaded state */
    int32_t force_list;           /* FORCE_LIST: 0, 2 or 3 */
    int32_t potential_flag;       /* POTENTIAL_FLAG: 0 LJ, 1 FENE polymer */
    int32_t rebuild_criteria;     /* REBUILD_CRITERIA: 0 vmax (Rapaport), 1 fixed, 2 exact displacement */
    int32_t fixed_rebuild;        /* FIXED_REBUILD period when rebuild_criteria = 1 */
    int32_t sLRC_flag;            /* SLRC_FLAG: long-range corrections on PE and P */
    int32_t precision;            /* FM_PRECISION_* */
    double k_c, R_0;              /* FENE_INFO spring constant and maximum extension */
    int32_t nlist_capacity;       /* neighbours per molecule reserved; 0 = automatic */
    int32_t threads_per_molecule; /* force kernel lanes per molecule; 0 = autotuned */
    int32_t integration_algorithm; /* INTEGRATION_ALGORITHM: 0 leap-frog (NVE), 1 velocity Verlet */
    int32_t list_build;           /* FM_LIST_BUILD_*: one warp per cell or per 2x2x2 cells (same rows) */
    int32_t solvent_flag;         /* SOLVENT_INFO with potential_flag 1: 0 all beads alike (WCA + bonds),
                                     1 Soddemann solvent of variable quality (force_list 3 only) */
    int32_t force_path;           /* FM_FORCE_PATH_*: how the neighbour-list force kernel reads partners
                                     (same pairs and results to FP64 rounding; only the speed differs) */
    double eps_pp, eps_ps, eps_ss; /* SOLVENT_INFO well depths: polymer-polymer, polymer-solvent,
                                      solvent-solvent (solvent_flag 1) */
} fm_params;

/* List build granularity: automatic (2x2x2 blocks below 8 molecules per
 * cell), one warp per cell, one warp per block of 2x2x2 cells.  The rows are
 * identical; only the speed differs. */
enum { FM_LIST_BUILD_AUTO = 0, FM_LIST_BUILD_CELLS = 1, FM_LIST_BUILD_BLOCKS = 2 };

/* Force kernel of the neighbour-list modes: automatic (the gather kernel),
 * one gather per list entry with threads_per_molecule lanes, or tiles -- one
 * CTA per block of 2x2x2 cells stages the block's 4x4x4-cell neighbourhood
 * (periodic images applied) in shared memory and the list holds 16-bit
 * offsets into that staging (half the list memory), read by
 * threads_per_molecule (4 or 8) lanes per molecule.  A handle on tiles leaves
 * them for the gather kernel when a neighbourhood outgrows the staging. */
enum { FM_FORCE_PATH_AUTO = 0, FM_FORCE_PATH_GATHER = 1, FM_FORCE_PATH_TILES = 2 };

/* Macroscopic properties of one record step, the columns of
 * results/macroscopic_properties (parallel_io.MPI2.f90:4589-4646) plus the
 * virial sum (simulation_record.f90:1205-1314). */
typedef struct fm_macro {
    int32_t iter;
    int32_t pad_;
    double simtime;
    double vsum;        /* sum of m v over all components */
    double mv2sum;      /* sum of m v^2 */
    double temperature; /* mv2sum / (3 N) */
    double kinenergy;   /* 0.5 mv2sum / N */
    double potenergy;   /* 0.5 sum PE_i / N + sLRC */
    double totenergy;
    double pressure;    /* rho/(3N) (mv2sum + virial/2) + P_sLRC */
    double virial;      /* sum of per-molecule virials */
} fm_macro;

typedef struct fm_handle fm_handle;

/* Geometry the reference derives from the parameters (no device needed):
 * ncells = floor(domain/(rcutoff+delta)), cellsidelength = domain/ncells,
 * rneighbr2 = (rcutoff + mean(delta))^2 with the FENE R_0 override, and
 * potshift = 4(rc^-12 - rc^-6).  With solvent_flag 1 a rneighbr below the
 * Soddemann range 1.5 raises rcutoff (and so the cells) to 1.5 and leaves
 * rneighbr2 as it is (:1871-1876).  Replaces set_parameters_cells
 * (setup_set_parameters.f90:1848-1903) and the potshift line (:1222).
 * Returns FM_ERR_FEWCELLS where the reference aborts. */
FM_API int fm_derive_geometry(const fm_params *p, int32_t ncells[3], double cellsidelength[3],
                       double *rneighbr2, double *rcutoff2, double *potshift);

/* Domain of an FCC start of nunits unit cells at a density
 * (set_parameters_global_domain, setup_set_parameters.f90:1545-1580). */
FM_API int fm_global_domain(const int32_t nunits[3], double density, double domain[3]);

/* ---- lifetime ------------------------------------------------------- */
/* Allocates device state for p->np molecules on the current CUDA device
 * (set_parameters_allocate, setup_set_parameters.f90:1248-1376). */
FM_API int fm_create(const fm_params *p, fm_handle **out);
FM_API int fm_destroy(fm_handle *h);
/* Orders all of the handle's device work on this cudaStream_t (NULL = the
 * legacy default stream). */
FM_API int fm_set_stream(fm_handle *h, void *cuda_stream);

/* ---- state transfer ------------------------------------------------- */
/* r, v (and optionally a) in the reference's column-major (3, n) layout,
 * i.e. r[3*i + k] = r(k+1, i+1).  glob_no (1-based) may be NULL: molecules
 * are then numbered 1..n in upload order.  The device copies are private to
 * the handle; host buffers are only read during the call. */
FM_API int fm_upload_state(fm_handle *h, int32_t n, const double *r, const double *v, const double *a,
                    const int32_t *glob_no);
/* Writes r, v, a (each may be NULL) back in upload order -- molecule i of
 * the upload is row i here whatever order the device keeps internally.
 * Blocks until the stream has drained. */
FM_API int fm_download_state(fm_handle *h, double *r, double *v, double *a, int32_t *glob_no);
/* FENE polymers (potential_flag 1): the reference's monomer record per
 * molecule in upload order -- chainID, subchainID and the four bin_bflag
 * words (polymer_info_MD; bin_bflag is (4, n)).  Call after fm_upload_state,
 * before fm_setup.  Bonds are then found while lists are built, as
 * check_update_adjacentbeadinfo does (linklist.f90:2542-2584).  With
 * solvent_flag 1, chainID 0 marks a solvent molecule (mark_chain_as_solvent,
 * modules.f90:681-707) and a pair's Soddemann well depth is eps_ss, eps_ps or
 * eps_pp by how many of the two are chain beads
 * (simulation_compute_forces_Soddemann_neigbr_halfint,
 * simulation_compute_forces.f90:793-888). */
FM_API int fm_upload_monomers(fm_handle *h, const int32_t *chainID, const int32_t *subchainID,
                              const int32_t *bin_bflag);
/* Mie_potential 1 (setup_set_parameters.f90:1208-1216): non-bonded pairs
 * use Mie_accijmag / Mie_energy (:149-204) and bonds harmonic_accijmag /
 * harmonic_energy (:384-437) with per-type-pair constants, and every
 * molecule has mass_lookup(moltype) (a = F/m; kinetic sums weighted by m,
 * simulation_record.f90:1236-1252).  The tables are the reference's own
 * lookup arrays after setup_mie_potential (:566-1092): ntypes x ntypes,
 * entry (i,j) at [(i-1) + ntypes*(j-1)], types 1-based; mass has ntypes
 * entries.  moltype(n) is in upload order.  With the Soddemann solvent
 * (solvent_flag 1) the WCA branch of its pair force is Mie_accijmag of the
 * pair's types (get_accijmag), its energy stays the LJ-WCA expression, the
 * pair accelerations are not divided by a mass and the harmonic bonds are
 * (simulation_compute_forces.f90:839-872, 752-754).  Call after
 * fm_upload_state (and fm_upload_monomers), before fm_setup.  No
 * counterpart entry point in the reference, whose tables are module
 * globals. */
#define FM_MIE_MAXTYPES 16
typedef struct fm_mie_tables {
    int32_t ntypes, pad_;
    const double *mass;                 /* mass_lookup(ntypes) */
    const double *epsilon;              /* epsilon_lookup */
    const double *lambdar, *lambdaa;    /* lambdar_lookup, lambdaa_lookup */
    const double *C, *alpha;            /* C_lookup, alpha_lookup */
    const double *potshift;             /* potshift_lookup */
    const double *k_harmonic, *r0;      /* k_lookup, r0_lookup (bonds) */
} fm_mie_tables;
FM_API int fm_set_mie(fm_handle *h, const fm_mie_tables *t, const int32_t *moltype);
/* angular_potential 1 (simulation_compute_forces_angular,
 * simulation_compute_forces.f90:981-1048, called at :257-259 with force_list
 * 3, potential_flag 1, solvent_flag 0): the bond-angle force of every middle
 * bead (funcy 2) and its two bonded partners, by the Mie types of the triple.
 * k_lookup, theta0_lookup: angular_k_lookup and angular_r0_lookup
 * (setup_set_parameters.f90:890-907), ntypes^3 each, (i,j,k) at
 * [(i-1) + ntypes*((j-1) + ntypes*(k-1))]; funcy per molecule (monomer%funcy).
 * The force is the reference's angular_harmonic_force (:441-489) with its i
 * and k in the order the reference's list build discovers the middle bead's
 * bonds, computed in the middle bead's frame (periodic images as the halo
 * copies form them) and applied to the three molecules.  No energy is
 * recorded (the reference records none).  Where the reference has no defined
 * result the step fails with FM_ERR_BOND: a middle bead without both bonds, or
 * a triple whose k_ijk < 1e-5.  After fm_set_mie, before fm_setup. */
FM_API int fm_set_angular(fm_handle *h, int32_t ntypes, const double *k_lookup, const double *theta0_lookup,
                          const int32_t *funcy);
/* Bonds of the last list build as (owner glob_no, partner glob_no, image
 * code) triplets, like fm_get_pair_list.  Test hook. */
FM_API int fm_get_bonds(fm_handle *h, int32_t *owner, int32_t *partner, int8_t *code, int64_t cap, int64_t *n);
/* Device pointers variant for callers that keep the state on the GPU:
 * d_r/d_v are (3, n) column-major FP64 device arrays, read or written on the
 * handle's stream without host staging. */
FM_API int fm_upload_state_device(fm_handle *h, int32_t n, const double *d_r, const double *d_v);
FM_API int fm_download_state_device(fm_handle *h, double *d_r, double *d_v, double *d_a);

/* ---- the drop-in subroutine mirrors (md.f90:143-163) ------------------ */
/* Initial cell binning, halo images, neighbour list, forces and record of
 * the uploaded state: assign_to_cell, messenger_updateborders(1),
 * assign_to_neighbourlist (md.f90:60-64) then simulation_compute_forces +
 * evaluate_macroscopic_properties (setup_initial_record.f90:88-89). */
FM_API int fm_setup(fm_handle *h);
/* simulation_move_particles_vv(pass_num), NVE (simulation_move_particles_vv.f90:64-69,132-135). */
FM_API int fm_move_vv(fm_handle *h, int32_t pass_num);
/* simulation_move_particles_lfv, NVE (simulation_move_particles_lfv.f90:81-92). */
FM_API int fm_move_lfv(fm_handle *h);
/* messenger_updateborders(rebuild) (messenger.MPI.f90:594-627).  Periodic
 * images are generated on the fly from their source molecule inside the
 * list-build and force kernels (x_img = x_src +/- domain, the same FP64 add),
 * so this call only validates the handle. */
FM_API int fm_update_borders(fm_handle *h, int32_t rebuild);
/* simulation_checkrebuild(rebuild) (simulation_checkrebuild.f90:17-148);
 * writes the 0/1 decision (blocks on the stream). */
FM_API int fm_check_rebuild(fm_handle *h, int32_t *rebuild);
/* linklist_deallocateall (linklist.f90:2872-2964): lists are overwritten in
 * place on the device, so this only validates the handle. */
FM_API int fm_linklist_deallocateall(fm_handle *h);
/* sendmols, single-rank form: periodic wrap r >= L/2 -> r-L, r < -L/2 -> r+L
 * (messenger.serial.f90:961-1028; messenger.MPI.f90:1383-1424). */
FM_API int fm_sendmols(fm_handle *h);
/* SORT_FLAG (setup_read_input.f90:812-827): sort_flag 0 off, 1 blocks in
 * x-fastest order, 2 blocks along a 3-D Hilbert curve; every sort_freq-th
 * rebuild; blocks of sortblocksize^3 cells.  Builds the block table Hcurve
 * (setup_set_parameters.f90:1140-1163) and resets the save variables of
 * sort_mols (nrebuilds 1, safety factors 1.5 and 5).  Call after
 * fm_upload_state.  Refused as the reference aborts: polymers, Mie, a
 * sort_flag other than 0..2; also a subdomain handle (its molecules are named
 * by global number, so their order carries nothing). */
FM_API int fm_set_sort(fm_handle *h, int32_t sort_flag, int32_t sort_freq, int32_t sortblocksize);
/* sort_mols (linklist.f90:2744-2869): on every sort_freq-th call, puts the
 * molecules in the order of their sort blocks' Hcurve numbers, stable within
 * a block; if a block holds more than ceiling((np/blocks) sf1 + sf2)
 * molecules it keeps the order and grows sf1 by 0.1 and sf2 by 5.  The order
 * is the one fm_download_state, fm_get_per_molecule and fm_get_pair_list
 * report in (global numbers move with their molecules); the device's own
 * layout stays in cell order.  The next cell sort orders each cell by the new
 * numbering, so list order and FP64 summation order follow it as they follow
 * the reference's array order.  Unlike the reference, a is permuted too (the
 * reference recomputes it before reading it).  fm_step runs it on the device
 * in each rebuild, after the periodic wrap.  With sort_flag 0 (the default)
 * it does nothing. */
FM_API int fm_sort_mols(fm_handle *h);
/* Counters of sort_mols: sorts done, sorts skipped by an overflowing block,
 * and its save variables nrebuilds, sf1, sf2.  Any output may be NULL. */
FM_API int fm_get_sort_state(fm_handle *h, int64_t *sorts, int64_t *skipped, int32_t *nrebuilds, double *sf1,
                             int32_t *sf2);
/* Hcurve for nblocks sort blocks per axis, x fastest, values 1..blocks:
 * sort_flag 1 numbers blocks in x-fastest order, 2 follows build_hilbert
 * (functions_lib.f90:2555-2604).  Host only; cap >= nblocks[0]*[1]*[2]. */
FM_API int fm_sort_table(int32_t sort_flag, const int32_t nblocks[3], int32_t *table, int64_t cap);
/* assign_to_cell (linklist.f90:2645-2679) as a counting sort: histogram,
 * exclusive scan, scatter.  Molecules are also re-ordered by cell on the
 * device (invisible through fm_download_state). */
FM_API int fm_assign_to_cell(fm_handle *h);
/* assign_to_neighbourlist (linklist.f90:2710-2741) for FORCE_LIST 2/3: the
 * pair set of assign_to_neighbourlist_halfint_opt (660-804) stored in both
 * directions, built from shared-memory cell tiles. */
FM_API int fm_assign_to_neighbourlist(fm_handle *h);
/* The rebuild branch of md_advance_vv (md.f90:150-157) as one call:
 * linklist_deallocateall, sendmols, sort_mols, assign_to_cell,
 * messenger_updateborders(1), assign_to_neighbourlist. */
FM_API int fm_rebuild_lists(fm_handle *h);
/* simulation_compute_forces (simulation_compute_forces.f90:182-275): zeroes
 * and recomputes a; per-molecule PE and virial when mod(iter,tplot) == 0. */
FM_API int fm_compute_forces(fm_handle *h);
/* evaluate_macroscopic_properties (simulation_record.f90:1205-1314) from the
 * sums of the last force evaluation that recorded PE and virial. */
FM_API int fm_evaluate_macroscopic_properties(fm_handle *h, fm_macro *out);
/* Sets the iteration counter (the reference's module global iter). */
FM_API int fm_set_iter(fm_handle *h, int32_t iter);
FM_API int fm_get_iter(fm_handle *h, int32_t *iter);

/* ---- the fused step loop -------------------------------------------- */
/* Runs nsteps iterations of md_advance_vv (md.f90:143-163) on the device --
 * move(1), rebuild check, [wrap, bin, list], forces, move(2), record -- or,
 * with integration_algorithm 0, of md_advance_lfv (md.f90:109-139): forces,
 * record, move, rebuild check, [wrap, bin, list].  The
 * rebuild decision is taken on the device, so the host never waits inside
 * the loop.  Returns after the work is queued unless blocking != 0; errors
 * detected on the device (escape, list overflow that cannot be resized, PE
 * blow-up) are reported by the next blocking call. */
FM_API int fm_step(fm_handle *h, int32_t nsteps, int32_t blocking);
/* Waits for queued work and returns the first device-side error, if any. */
FM_API int fm_sync(fm_handle *h);

/* ---- results -------------------------------------------------------- */
/* Records (one per tplot step) produced since the previous call, oldest
 * first.  *n receives how many were written (at most cap). */
FM_API int fm_get_records(fm_handle *h, fm_macro *out, int32_t cap, int32_t *n);
/* Per-molecule potenergymol and virialmol of the last recording force
 * evaluation, in upload order. */
FM_API int fm_get_per_molecule(fm_handle *h, double *potenergymol, double *virialmol);
/* Neighbour pairs as (owner glob_no, partner glob_no, image code) triplets,
 * image code = (sx+1) + 3(sy+1) + 9(sz+1) for the domain shift of the
 * partner, 13 = no shift.  Both directions of every pair are listed.  *n is
 * the total; at most cap triplets are written.  Test hook. */
FM_API int fm_get_pair_list(fm_handle *h, int32_t *owner, int32_t *partner, int8_t *code, int64_t cap,
                     int64_t *n);
/* Order-independent 64-bit digest of the canonical pair set (a sum of
 * mixed hashes of (min gid, max gid) for unshifted pairs and of
 * (owner, partner, code) for image pairs); matches the oracle's digest of
 * the reference half list. */
FM_API int fm_pair_digest(fm_handle *h, uint64_t *digest, int64_t *npairs);
/* Force-kernel lanes per molecule in use (fixed, or chosen by the autotuner at fm_setup). */
FM_API int fm_get_threads_per_molecule(fm_handle *h, int32_t *tpm);
/* Force kernel in use (FM_FORCE_PATH_GATHER or FM_FORCE_PATH_TILES; a handle
 * leaves the tiled path when a staged neighbourhood outgrows shared memory),
 * and the staged-candidate capacity of a block on the tiled path (0 otherwise).
 * No counterpart in the reference: a diagnostic of this implementation. */
FM_API int fm_get_force_path(fm_handle *h, int32_t *path, int32_t *tile_capacity);
/* Counters: rebuilds done, neighbour capacity in use, largest list seen. */
FM_API int fm_get_counters(fm_handle *h, int64_t *rebuilds, int32_t *nlist_capacity, int32_t *max_neighbours);

/* ---- restart files and keyword input (host only, no device needed) ---- */
#define FM_RESTART_MAXPROC 4096

/* Header of a final_state restart file (parallel_io.MPI2.f90:1650-1700). */
typedef struct fm_restart_header {
    int32_t globalnp;
    int32_t initialnunits[3];
    int32_t nsteps;              /* Nsteps, or iter when written before the end */
    int32_t tplot;
    int32_t seed[2];
    int32_t periodic[3];
    int32_t potential_flag, rtrue_flag, solvent_flag, nmonomers;
    int32_t npx, npy, npz, nproc;
    int32_t mie_potential, global_numbering;
    int64_t header_pos;          /* byte offset of the header (read only) */
    double globaldomain[3];
    double density, rcutoff, delta_t, elapsedtime, simtime, k_c, R_0, eps_pp, eps_ps, eps_ss;
    double delta_rneighbr;       /* delta_rneighbr(1) */
    int32_t procnp[FM_RESTART_MAXPROC];
    int32_t proctethernp[FM_RESTART_MAXPROC];
} fm_restart_header;

/* Reads a final_state file (the body layout of parallel_io_final_state,
 * parallel_io.MPI2.f90:1495-1726; global coordinates).  With r and v NULL
 * only the header is read.  Arrays hold cap >= globalnp molecules: r, v,
 * rtether, rtrue are (3, n) column-major, monomer is (8, n); any may be NULL.
 * glob_no is 1..n when the file has no global numbering; rtether is 0 for
 * untethered molecules. */
FM_API int fm_read_final_state(const char *path, fm_restart_header *hdr, int32_t cap, double *r, double *v,
                               int32_t *tag, double *rtether, int32_t *glob_no, double *rtrue, int32_t *moltype,
                               double *monomer);
/* Writes a final_state file byte-compatible with the reference's. */
FM_API int fm_write_final_state(const char *path, const fm_restart_header *hdr, const double *r, const double *v,
                                const int32_t *tag, const double *rtether, const int32_t *glob_no,
                                const double *rtrue, const int32_t *moltype, const double *monomer);

/* Hot-path subset of the keyword input file (setup_read_input.f90, keyword
 * search of functions_lib.f90:1139-1193). */
typedef struct fm_input {
    int32_t ensemble, integration_algorithm, force_list, potential_flag;
    int32_t nsteps, tplot, rebuild_criteria, fixed_rebuild;
    int32_t initialnunits[3], periodic[3];
    int32_t sort_flag, global_numbering, pressure_outflag, sLRC_flag, mie_potential, nmonomers, nthermo;
    int32_t solvent_flag;        /* SOLVENT_INFO [1] */
    double density, rcutoff, inputtemperature, delta_t, delta_rneighbr[3], k_c, R_0;
    double tethereddisttop[3], tethereddistbottom[3], thermstattop[3], thermstatbottom[3];
    double slidedisttop[3], slidedistbottom[3], fixdisttop[3], fixdistbottom[3], wallslidev[3];
    double teth_k[3];            /* TETHERCOEFFICIENTS k2, k4, k6 */
    double thermostattemperature[2];
    double targetconc;           /* FENE_SOLUTION [5] */
    double eps_pp, eps_ps, eps_ss; /* SOLVENT_INFO [2-4] when solvent_flag is 1 */
    int32_t sort_freq, sortblocksize; /* SORT_FLAG [2-3] (for fm_set_sort) */
} fm_input;

FM_API int fm_read_input(const char *path, fm_input *in);

/* ---- multi-job engine: batched replicas and served jobs ---------------- */
/* No single counterpart in the reference, which runs one system per MPI job:
 * the engine keeps many independent systems resident on one GPU and advances
 * all of them one step per tick with the same kernels as above (per-job
 * geometry, iteration counter, rebuild state and status).  Batching submits
 * all replicas and runs until drained; serving submits jobs as they arrive
 * and calls fm_engine_step_chunk in a loop -- jobs are admitted whenever a
 * slot and enough arena memory (molecules, cells, neighbour rows) are free,
 * and retired as soon as they finish. */
typedef struct fm_engine fm_engine;

typedef struct fm_engine_params {
    int64_t max_molecules;        /* molecule arena: sum of resident job sizes */
    int64_t max_cells;            /* extended-cell arena */
    int64_t max_list_entries;     /* neighbour-row arena (entries) */
    int32_t max_slots;            /* jobs resident at once */
    int32_t precision;            /* FM_PRECISION_* for every job */
    int32_t threads_per_molecule; /* 0 = autotuned on the first resident jobs */
    int32_t ticks_per_chunk;      /* most steps per graph launch between admission points (a launch
                                     ends earlier when a job finishes while others are queued) */
    int32_t keep_states;          /* keep final r, v of finished jobs for fm_engine_job_state */
    int32_t list_build;           /* FM_LIST_BUILD_*: the list build's tile, one cell or 2x2x2 cells per
                                     warp (same rows); AUTO = chosen by timing the resident jobs */
    double delta_t;               /* DELTA_T shared by every job */
} fm_engine_params;

/* Molecular tags (the reference's modules.f90:79-86). */
#define FM_TAG_FREE 0
#define FM_TAG_FIXED 1
#define FM_TAG_FIXED_SLIDE 2
#define FM_TAG_TETH 3
#define FM_TAG_THERMO 4
#define FM_TAG_TETH_THERMO 5
#define FM_TAG_TETH_SLIDE 6
#define FM_TAG_TETH_THERMO_SLIDE 7

typedef struct fm_job {
    int32_t np;
    int32_t tplot;
    double domain[3];
    double density;
    double rcutoff;
    double delta_rneighbr[3];
    int32_t nsteps;                 /* NSTEPS of this job */
    int32_t initialstep;
    int32_t integration_algorithm;  /* 0 leap-frog (tags allowed), 1 velocity Verlet */
    int32_t ensemble;               /* 0 NVE, 6 tag_move */
    int32_t force_list;             /* 0 all pairs (any box), 2/3 neighbour list (>= 3 cells) */
    int32_t pressure_outflag;       /* 1: time-average the virial pressure tensor over record steps */
    int32_t nthermo;                /* thermostat regions: 0, 1, or 2 split at y = 0 */
    int32_t rebuild_criteria;       /* 0 vmax, 1 fixed */
    int32_t fixed_rebuild;
    int32_t nlist_capacity;         /* neighbour slots per molecule; 0 = automatic */
    double thermostat_temperature[2];
    double teth_k2, teth_k4, teth_k6; /* TETHERCOEFFICIENTS */
} fm_job;

typedef struct fm_job_result {
    int64_t job_id;
    int32_t status;          /* FM_OK or the error the job ended with */
    int32_t nsamples;        /* record steps averaged into ptensor */
    int32_t final_iter;
    int32_t rebuilds;
    int32_t retries;         /* re-admissions after neighbour-list overflow */
    int32_t pad_;
    double ptensor[9];       /* time-averaged sum(v v + r f / 2)/V over record steps, row-major */
    fm_macro last;           /* the last record */
    double submit_time, admit_time, finish_time;  /* host seconds (steady clock) */
} fm_job_result;

FM_API int fm_engine_create(const fm_engine_params *p, fm_engine **out);
FM_API int fm_engine_destroy(fm_engine *e);
FM_API int fm_engine_set_stream(fm_engine *e, void *cuda_stream);
/* Queues a job: r, v are (3, np) column-major; tag (np), rtether and slidev
 * ((3, np)) may be NULL.  The arrays are copied; returns the job id.  A job
 * keeps its molecules in submission order: sort_mols (fm_set_sort) is a
 * single-system feature, so a job's results come back in the order it was
 * submitted in, whatever the deck's SORT_FLAG. */
FM_API int fm_engine_submit(fm_engine *e, const fm_job *job, const double *r, const double *v, const int32_t *tag,
                            const double *rtether, const double *slidev, int64_t *job_id);
/* One admission point (retire finished jobs, admit queued ones that fit)
 * followed by one chunk of ticks: one graph launch whose ticks loop on the
 * device, min(ticks_per_chunk, 32) per iteration, until no job is left
 * running, ticks_per_chunk ticks have run, a job has failed, or -- while
 * jobs wait in the queue -- a job has finished; reports how many jobs are
 * resident and queued afterwards. */
FM_API int fm_engine_step_chunk(fm_engine *e, int32_t *resident, int32_t *queued);
/* Chunks until nothing is resident or queued (max_chunks <= 0: no limit). */
FM_API int fm_engine_run(fm_engine *e, int32_t max_chunks);
/* Finished jobs' results, oldest first (each returned once). */
FM_API int fm_engine_take_results(fm_engine *e, fm_job_result *out, int32_t cap, int32_t *n);
/* Final r, v of a finished job in its upload order (keep_states = 1). */
FM_API int fm_engine_job_state(fm_engine *e, int64_t job_id, double *r, double *v);
FM_API int fm_engine_counters(fm_engine *e, int64_t *ticks, int64_t *molecule_steps, int32_t *threads_per_molecule,
                              int64_t *launches);
/* The autotuner's choices: force-kernel lanes per molecule, and the list
 * build's tile -- jobs with fewer than `blocks_below` molecules per cell are
 * built by 2x2x2-cell blocks, the rest one cell per warp (0: every job by
 * cells).  Both are chosen on the first resident jobs by timing the force
 * kernel and the list build over them (no counterpart in the reference). */
FM_API int fm_engine_tuning(fm_engine *e, int32_t *threads_per_molecule, double *blocks_below);

/* ---- instrumentation -------------------------------------------------- */
/* When enabled, every force-kernel launch is bracketed by CUDA events on the
 * handle's stream; fm_get_force_kernel_time returns the summed device time
 * (ms) and the number of launches since it was last read. */
FM_API int fm_force_kernel_timing(fm_handle *h, int32_t enable);
FM_API int fm_get_force_kernel_time(fm_handle *h, double *ms, int64_t *launches);
/* PRESSURE_OUTFLAG 1, the full-domain virial stress (pressure_averaging and
 * cumulative_pressure case 1, simulation_record.f90:3103-3220).  On every
 * record step P = sum_i (v_i v_i + rf_i / 2) / volume is added to a running
 * sum, with rf_i = sum of accijmag rij rij over i's pair and bond terms
 * (pressure_tensor_forces, :6239-6256: the LJ/Mie half- and full-list pairs
 * and the FENE/harmonic bonds; the all-pairs and Soddemann routines add none,
 * as in the reference) and v the record velocity (leap-frog: v + a dt/2).
 * Setting the flag clears the sum.  fm_get_pressure_tensor gives the mean of
 * the samples (row-major 3x3) and their count, and clears the sum when
 * `reset` is non-zero -- Pxy / Nstress_ave when read every Nstress_ave
 * samples. */
FM_API int fm_set_pressure_outflag(fm_handle *h, int32_t flag);
FM_API int fm_get_pressure_tensor(fm_handle *h, double P[9], int32_t *nsamples, int32_t reset);
/* Kernels this handle has launched since creation: the host's launches plus
 * the rebuild kernels that the device ran inside the rebuild graph of a step
 * (waits for the handle's stream). */
FM_API int fm_get_launch_count(fm_handle *h, int64_t *launches);

/* ---- forces without device allocation -------------------------------- */
/* No counterpart in the reference (Flowmol always owns its arrays).  For
 * callers that cannot call cudaMalloc -- a host code whose device memory is
 * all handed out by its own pool or framework, or a loop that must not take
 * the device-wide synchronisation an allocation can imply -- this computes
 * the same LJ forces, per-molecule PE and virial as fm_setup/fm_compute_forces
 * for positions already on the device, without allocating: its scratch is one
 * fixed __device__ array (about 3 MB, resident on every GPU that loads the
 * library until exit) shared by all calls.  d_r, d_a are (3, n) column-major
 * FP64 device arrays; d_potenergymol and d_virialmol (n) may be NULL.  Uses
 * p->domain, rcutoff, delta_rneighbr, precision.  Positions outside
 * [-L/2, L/2) are wrapped by one period on a private copy first (d_r is not
 * written), so the result is fm_setup's for the wrapped positions.  Limits:
 * n <= FM_NOALLOC_MAX_MOLECULES and (ncells+2)^3 <= FM_NOALLOC_MAX_CELLS,
 * else FM_ERR_ARG.  The first call on a device looks up the array's device
 * address, so make it before any stream capture; the address is kept, so do
 * not call this on a device after a cudaDeviceReset of that device.  Calls
 * that overlap on the GPU race on the shared scratch.  Every call reads a
 * status word back to the host and waits for cuda_stream to drain before it
 * returns. */
#define FM_NOALLOC_MAX_MOLECULES 65536
#define FM_NOALLOC_MAX_CELLS 32768
FM_API int fm_compute_forces_noalloc(const fm_params *p, int32_t n, const double *d_r, double *d_a,
                                     double *d_potenergymol, double *d_virialmol, void *cuda_stream);
/* Message of the last failing fm_compute_forces_noalloc call on this thread. */
FM_API int fm_noalloc_last_error(char *buf, int32_t len);

/* ---- spatial decomposition: one rank's subdomain ---------------------- */
/* The reference's MPI build splits the box over a process grid
 * (messenger_init, messenger.MPI.f90:222-550), refreshes every rank's halo of
 * the neighbours' boundary cells each step (messenger_updateborders,
 * :594-628, faces/edges/corners :882-1380) and moves molecules to the rank
 * whose subdomain they entered on rebuilds (sendmols, :1383-1421).  Here a
 * subdomain is a block of the UNDIVIDED system's cells in global coordinates:
 * interior cells origin .. origin + ncells_local - 1 (0-based, per axis) of
 * the ncells_global that fm_derive_geometry gives for p (p->np is the whole
 * system's count).  Molecules are binned, ordered (by global number) and
 * paired exactly as in the undivided system, so forces and trajectories are
 * bit-identical to one fm_handle over the whole box; records differ only in
 * the order the ranks' sums are added.  Scope: force_list 2/3, LJ/WCA
 * (potential_flag 0), velocity Verlet, rebuild_criteria 0/1.
 *
 * The caller moves the data between ranks: flat FP64 record buffers in device
 * memory (FM_DD_MREC doubles per migrating molecule, FM_DD_HREC per halo
 * copy, 3 per refreshed position), grouped by destination rank in rank
 * order, with counts per destination (an all-to-all; NCCL or gloo).  A
 * rebuild (at setup: wrap = 0; on a step: wrap = 1):
 *   fm_dd_classify(counts) -> all-to-all counts -> fm_dd_pack_emigrants
 *   -> all-to-all records -> fm_dd_immigrate -> fm_dd_halo_counts(counts)
 *   -> all-to-all counts -> fm_dd_pack_halo -> all-to-all records
 *   -> fm_dd_receive_halo (counting sort + neighbour rows).
 * Between rebuilds the halo positions are refreshed from lists the caller
 * derives from fm_dd_cell_starts and the plan: fm_dd_gather_positions ->
 * all-to-all -> fm_dd_scatter_positions.  A velocity-Verlet step:
 * fm_dd_vmax2 -> max over ranks -> fm_dd_decide -> (rebuild | refresh) ->
 * fm_dd_forces(mode 2) -> on record steps fm_dd_sums -> sum over ranks ->
 * fm_dd_macro.  No call here communicates. */
#define FM_DD_MREC 10
#define FM_DD_HREC 5
#define FM_DD_NSUMS 11 /* pe, virial, mv2, vsum, max pe, 6 pressure terms (0 here) */
FM_API int fm_dd_create(const fm_params *p, const int32_t ncells_global[3], const int32_t origin[3],
                        const int32_t ncells_local[3], int32_t capacity, fm_handle **out);
/* The process grid (rank = (px dims[1] + py) dims[2] + pz, as MPI_Cart_create
 * numbers it), the process coordinate owning each global interior cell
 * (owner_axis: x cells, then y, then z), and per local extended cell c the
 * needs [need_off[c], need_off[c+1]): the rank whose halo holds it, the image
 * code it is seen with ((sx+1) | (sy+1)<<2 | (sz+1)<<4) and that rank's local
 * halo cell. */
FM_API int fm_dd_set_plan(fm_handle *h, int32_t rank, const int32_t dims[3], const int32_t *owner_axis,
                          const int32_t *need_off, const int32_t *need_rank, const int32_t *need_code,
                          const int32_t *need_cell);
/* The rank's molecules (r, v host (3, n) column-major; gid 0-based global numbers). */
FM_API int fm_dd_upload(fm_handle *h, int32_t n, const double *r, const double *v, const int32_t *gid);
FM_API int fm_dd_classify(fm_handle *h, int32_t wrap, int32_t *counts);
FM_API int fm_dd_pack_emigrants(fm_handle *h, double *d_send);
FM_API int fm_dd_immigrate(fm_handle *h, const double *d_recv, int32_t n);
FM_API int fm_dd_halo_counts(fm_handle *h, int32_t *counts);
FM_API int fm_dd_pack_halo(fm_handle *h, double *d_send);
FM_API int fm_dd_receive_halo(fm_handle *h, const double *d_recv, int32_t n);
FM_API int fm_dd_counts(fm_handle *h, int32_t *n_owned, int32_t *n_halo);
/* ncells + 1 starts of the local extended cells after the last sort. */
FM_API int fm_dd_cell_starts(fm_handle *h, int32_t *starts);
FM_API int fm_dd_gather_positions(fm_handle *h, const int32_t *d_idx, const int8_t *d_code, int32_t n,
                                  double *d_out);
FM_API int fm_dd_scatter_positions(fm_handle *h, const int32_t *d_idx, const double *d_in, int32_t n);
/* Velocity-Verlet pass 1 in place (the first step after a rebuild at setup). */
FM_API int fm_dd_move1(fm_handle *h);
FM_API int fm_dd_vmax2(fm_handle *h, uint64_t *vmax2);
/* simulation_checkrebuild with the ranks' largest |v|^2 (bits of the double);
 * flip = 1 when the last force call moved the molecules (mode 2). */
FM_API int fm_dd_decide(fm_handle *h, uint64_t vmax2_global, int32_t iter, int32_t flip, int32_t *rebuild);
/* Forces of the owned molecules: mode 0 forces only, 1 + move(2), 2 + move(2)
 * and the next move(1); record = 1 on tplot steps (partials for fm_dd_sums). */
FM_API int fm_dd_forces(fm_handle *h, int32_t iter, int32_t record, int32_t mode);
FM_API int fm_dd_sums(fm_handle *h, double *sums);
FM_API int fm_dd_macro(fm_handle *h, const double *sums, int32_t iter, double simtime, fm_macro *out);
/* The owned molecules in slot order (r, v (3, n) column-major, gid). */
FM_API int fm_dd_download(fm_handle *h, int32_t cap, int32_t *n_owned, double *r, double *v, int32_t *gid);
/* Neighbour rows as (owner, partner) global numbers and the partner's local
 * extended cell (a halo cell's image code is the plan's), for tests. */
FM_API int fm_dd_pair_list(fm_handle *h, int32_t *owner, int32_t *partner, int32_t *partner_cell, int64_t cap,
                           int64_t *n_out);

/* ---- errors --------------------------------------------------------- */
/* Copies the message of the last failing call on this thread. */
FM_API int fm_last_error(char *buf, int32_t len);

#ifdef __cplusplus
}
#endif
#endif /* FLOWMOL_B200_H */
