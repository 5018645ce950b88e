// fm_noalloc.cu -- LJ forces for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a host code whose
// device memory is handed out by its own pool or framework (every byte is
// already reserved, and a foreign allocation would break its budget), or a
// driver loop that must not take the device-wide synchronisation that
// cudaMalloc/cudaFree can imply.  fm_compute_forces_noalloc serves them: it
// evaluates the same forces as fm_setup / fm_compute_forces (cell binning by
// counting sort, then every pair within rcutoff over the 27-cell stencil with
// the reference's periodic-image roundings), but its scratch -- cell counts,
// cell starts, the cell-ordered copy of the positions -- lives in one
// file-scope __device__ array of fixed size instead of memory allocated per
// handle.  It calls no cudaMalloc, cudaFree or allocating library routine.
//
// Positions outside [-L/2, L/2) are wrapped by one period on a private copy
// before binning (the wrap sendmols applies at a rebuild), so the forces are
// those fm_setup computes for the wrapped positions.
//
// Limits: at most FM_NOALLOC_MAX_MOLECULES molecules and
// FM_NOALLOC_MAX_CELLS extended cells ((ncells+2)^3); larger inputs are
// rejected with FM_ERR_ARG.  The array is about 3 MB and stays resident on
// every GPU that loads the library until the process exits.  All calls share
// it: two calls that overlap on the GPU (different streams, or different
// host threads on one device) race and corrupt each other's results.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "flowmol_b200.h"

namespace {

constexpr int NA_MAX_N = FM_NOALLOC_MAX_MOLECULES;
constexpr int NA_MAX_CELLS = FM_NOALLOC_MAX_CELLS;

// Scratch layout (byte offsets; every block 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t OFF_STATUS = 0;                                             // uint32 status + pad
constexpr size_t OFF_COUNT = 256;                                            // int32[NA_MAX_CELLS]
constexpr size_t OFF_START = OFF_COUNT + align256(4ull * NA_MAX_CELLS);      // int32[NA_MAX_CELLS+1]
constexpr size_t OFF_CELLOF = OFF_START + align256(4ull * (NA_MAX_CELLS + 1));  // int32[NA_MAX_N]
constexpr size_t OFF_SPOS = OFF_CELLOF + align256(4ull * NA_MAX_N);          // double4[NA_MAX_N]
constexpr size_t SCRATCH_BYTES = OFF_SPOS + align256(32ull * NA_MAX_N);

__device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

struct NaGeom {
    int n;
    double L[3], hd[3], cs[3];
    int ne[3];
    int ncell;
    double rc2, potshift;
    int precision;
    int want_pe, want_vir;
};

struct NaScratch {
    unsigned int *status;
    int *count, *start, *cell_of;
    double4 *spos;  // cell-ordered x, y, z and the molecule's original index in w
};

__host__ NaScratch carve(unsigned char *base)
{
    NaScratch s;
    s.status = reinterpret_cast<unsigned int *>(base + OFF_STATUS);
    s.count = reinterpret_cast<int *>(base + OFF_COUNT);
    s.start = reinterpret_cast<int *>(base + OFF_START);
    s.cell_of = reinterpret_cast<int *>(base + OFF_CELLOF);
    s.spos = reinterpret_cast<double4 *>(base + OFF_SPOS);
    return s;
}

__device__ __forceinline__ double n2(double x, double y, double z)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

__device__ __forceinline__ int na_bin(double x, double hd, double cs, int ne, bool &bad)
{
    double q = __ddiv_rn(__dadd_rn(x, hd), cs);
    if (!(q == q)) { bad = true; return 0; }
    int c = __double2int_ru(q);
    if (c < 0 || c > ne - 1) { bad = true; c = c < 0 ? 0 : ne - 1; }
    return c;
}

__global__ void k_na_zero(NaGeom g, NaScratch s)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < g.ncell) s.count[c] = 0;
    if (c == 0) *s.status = 0u;
}

// One period of wrap, as sendmols does at a rebuild (r >= L/2 -> r - L,
// r < -L/2 -> r + L): the caller's positions are left as they are and the
// wrapped copy is what gets binned and paired.
__device__ __forceinline__ double na_wrap(double x, double hd, double L)
{
    if (x >= hd) x = __dsub_rn(x, L);
    if (x < -hd) x = __dadd_rn(x, L);
    return x;
}

__global__ void k_na_bin(NaGeom g, NaScratch s, const double *r3)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    bool bad = false;
    const double x = na_wrap(r3[3 * (size_t)i], g.hd[0], g.L[0]);
    const double y = na_wrap(r3[3 * (size_t)i + 1], g.hd[1], g.L[1]);
    const double z = na_wrap(r3[3 * (size_t)i + 2], g.hd[2], g.L[2]);
    int cx = na_bin(x, g.hd[0], g.cs[0], g.ne[0], bad);
    int cy = na_bin(y, g.hd[1], g.cs[1], g.ne[1], bad);
    int cz = na_bin(z, g.hd[2], g.cs[2], g.ne[2], bad);
    if (bad) atomicOr(s.status, 1u);
    int c = cx + g.ne[0] * (cy + g.ne[1] * cz);
    s.cell_of[i] = c;
    atomicAdd(&s.count[c], 1);
}

constexpr int NA_SCAN = 1024;
__global__ void __launch_bounds__(NA_SCAN) k_na_scan(NaGeom g, NaScratch s)
{
    __shared__ int ws[32];
    const int nc = g.ncell;
    const int per = (nc + NA_SCAN - 1) / NA_SCAN;
    const int b = threadIdx.x * per, e = min(b + per, nc);
    int local = 0;
    for (int c = b; c < e; c++) local += s.count[c];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[w] = incl;
    __syncthreads();
    if (w == 0) {
        int v = ws[lane], vi = v;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, vi, o);
            if (lane >= o) vi += t;
        }
        ws[lane] = vi - v;
    }
    __syncthreads();
    int run = ws[w] + incl - local;
    for (int c = b; c < e; c++) {
        int k = s.count[c];
        s.start[c] = run;
        s.count[c] = 0;
        run += k;
    }
    if (threadIdx.x == NA_SCAN - 1) s.start[nc] = run;
}

__global__ void k_na_scatter(NaGeom g, NaScratch s, const double *r3)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    int c = s.cell_of[i];
    int slot = s.start[c] + atomicAdd(&s.count[c], 1);
    s.spos[slot] = make_double4(na_wrap(r3[3 * (size_t)i], g.hd[0], g.L[0]),
                                na_wrap(r3[3 * (size_t)i + 1], g.hd[1], g.L[1]),
                                na_wrap(r3[3 * (size_t)i + 2], g.hd[2], g.L[2]), (double)i);
}

// Deterministic in-cell order (by original index).
__global__ void k_na_sort(NaGeom g, NaScratch s)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.ncell) return;
    int b = s.start[c], e = s.start[c + 1];
    for (int x = b + 1; x < e; x++) {
        double4 key = s.spos[x];
        int y = x - 1;
        while (y >= b && s.spos[y].w > key.w) {
            s.spos[y + 1] = s.spos[y];
            y--;
        }
        s.spos[y + 1] = key;
    }
}

__device__ __forceinline__ bool halo_axis(int x, int ne) { return x == 0 || x == ne - 1; }

// One thread per molecule (cell order): every candidate of the 27 cells
// around its cell that are not both halo with it -- real molecules of the
// cell, plus, for a halo cell, the images of the interior cell on the far
// side shifted by +/-domain -- tested against rcutoff2 in FP64.
template <int PREC>
__global__ void k_na_force(NaGeom g, NaScratch s, double *a3, double *pe_out, double *vir_out)
{
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= g.n) return;
    const double4 pi = s.spos[slot];
    const int i = (int)pi.w;
    const int c = s.cell_of[i];
    const int cx = c % g.ne[0], cy = (c / g.ne[0]) % g.ne[1], cz = c / (g.ne[0] * g.ne[1]);
    const bool chalo = halo_axis(cx, g.ne[0]) || halo_axis(cy, g.ne[1]) || halo_axis(cz, g.ne[2]);
    double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0, vir = 0.0;
    for (int q = 0; q < 27; q++) {
        int x2 = cx + q % 3 - 1, y2 = cy + (q / 3) % 3 - 1, z2 = cz + q / 9 - 1;
        if (x2 < 0 || y2 < 0 || z2 < 0 || x2 >= g.ne[0] || y2 >= g.ne[1] || z2 >= g.ne[2]) continue;
        bool h2 = halo_axis(x2, g.ne[0]) || halo_axis(y2, g.ne[1]) || halo_axis(z2, g.ne[2]);
        if (chalo && h2) continue;
        for (int pass = 0; pass < (h2 ? 2 : 1); pass++) {
            int sx = 0, sy = 0, sz = 0, src = x2 + g.ne[0] * (y2 + g.ne[1] * z2);
            if (pass == 1) {
                sx = x2 == 0 ? -1 : (x2 == g.ne[0] - 1 ? 1 : 0);
                sy = y2 == 0 ? -1 : (y2 == g.ne[1] - 1 ? 1 : 0);
                sz = z2 == 0 ? -1 : (z2 == g.ne[2] - 1 ? 1 : 0);
                int xs = x2 == 0 ? g.ne[0] - 2 : (x2 == g.ne[0] - 1 ? 1 : x2);
                int ys = y2 == 0 ? g.ne[1] - 2 : (y2 == g.ne[1] - 1 ? 1 : y2);
                int zs = z2 == 0 ? g.ne[2] - 2 : (z2 == g.ne[2] - 1 ? 1 : z2);
                src = xs + g.ne[0] * (ys + g.ne[1] * zs);
            }
            const int b = s.start[src], e = s.start[src + 1];
            for (int j = b; j < e; j++) {
                if (j == slot && pass == 0) continue;
                double4 pj = s.spos[j];
                double xj = sx ? __dadd_rn(pj.x, sx > 0 ? g.L[0] : -g.L[0]) : pj.x;
                double yj = sy ? __dadd_rn(pj.y, sy > 0 ? g.L[1] : -g.L[1]) : pj.y;
                double zj = sz ? __dadd_rn(pj.z, sz > 0 ? g.L[2] : -g.L[2]) : pj.z;
                double dx = __dsub_rn(pi.x, xj), dy = __dsub_rn(pi.y, yj), dz = __dsub_rn(pi.z, zj);
                double r2 = n2(dx, dy, dz);
                if (r2 < g.rc2) {
                    if (PREC == 0) {
                        const double sv = 1.0 / r2, s2 = sv * sv, s4 = s2 * s2;
                        const double acc = 48.0 * (s4 * s2 * sv - 0.5 * s4);
                        fx += acc * dx; fy += acc * dy; fz += acc * dz;
                        const double s3 = s2 * sv;
                        pe += 4.0 * (s3 * s3 - s3) - g.potshift;
                        vir += acc * r2;
                    } else {
                        // the precision form of the main force kernel: FP32 pair
                        // magnitude, scaled by the FP64 rij, sums in FP64
                        const float sv = __frcp_rn((float)r2), s2 = sv * sv, s4 = s2 * s2;
                        const double acc = (double)(48.0f * (s4 * s2 * sv - 0.5f * s4));
                        fx = fma(acc, dx, fx); fy = fma(acc, dy, fy); fz = fma(acc, dz, fz);
                        const float s3 = s2 * sv, s6 = s3 * s3;
                        pe += (double)(4.0f * (s6 - s3)) - g.potshift;
                        vir += acc * r2;
                    }
                }
            }
        }
    }
    a3[3 * (size_t)i] = fx; a3[3 * (size_t)i + 1] = fy; a3[3 * (size_t)i + 2] = fz;
    if (pe_out) pe_out[i] = pe;
    if (vir_out) vir_out[i] = vir;
}

thread_local std::string g_na_error;
std::mutex g_na_mutex;
unsigned char *g_na_base[256];  // device address of the scratch array, per device ordinal

int na_fail(int code, const std::string &msg)
{
    g_na_error = msg;
    return code;
}

}  // namespace

// Message of the last failing fm_compute_forces_noalloc call on this thread.
extern "C" int fm_noalloc_last_error(char *buf, int32_t len)
{
    if (!buf || len <= 0) return FM_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", g_na_error.c_str());
    return FM_OK;
}

extern "C" int fm_compute_forces_noalloc(const fm_params *p, int32_t n, const double *d_r, double *d_a,
                                         double *d_potenergymol, double *d_virialmol, void *cuda_stream)
{
    if (!p || !d_r || !d_a) return na_fail(FM_ERR_ARG, "null argument");
    if (n != p->np || n <= 0) return na_fail(FM_ERR_ARG, "n must equal params->np and be > 0");
    if (n > NA_MAX_N)
        return na_fail(FM_ERR_ARG, "fm_compute_forces_noalloc: " + std::to_string(n) +
                                       " molecules exceed the fixed scratch limit of " + std::to_string(NA_MAX_N));
    if (!(p->rcutoff > 0.0)) return na_fail(FM_ERR_ARG, "rcutoff must be > 0");
    if (p->precision != FM_PRECISION_FP64 && p->precision != FM_PRECISION_FP32)
        return na_fail(FM_ERR_ARG, "precision must be FM_PRECISION_FP64 or FM_PRECISION_FP32");
    NaGeom g{};
    g.n = n;
    for (int k = 0; k < 3; k++) {
        if (!(p->domain[k] > 0.0)) return na_fail(FM_ERR_ARG, "domain must be > 0");
        int nc = (int)std::floor(p->domain[k] / (p->rcutoff + p->delta_rneighbr[k]));  // set_parameters_cells
        if (nc < 3) return na_fail(FM_ERR_FEWCELLS, "domain should have at least 3 cells in x, y and z");
        g.L[k] = p->domain[k];
        g.hd[k] = 0.5 * p->domain[k];
        g.cs[k] = p->domain[k] / (double)nc;
        g.ne[k] = nc + 2;
    }
    long long ncell = (long long)g.ne[0] * g.ne[1] * g.ne[2];
    if (ncell > NA_MAX_CELLS)
        return na_fail(FM_ERR_ARG, "fm_compute_forces_noalloc: " + std::to_string(ncell) +
                                       " extended cells exceed the fixed scratch limit of " +
                                       std::to_string(NA_MAX_CELLS));
    g.ncell = (int)ncell;
    g.rc2 = p->rcutoff * p->rcutoff;
    {
        double rc = p->rcutoff, r3 = rc * rc * rc, r6 = r3 * r3, r12 = r6 * r6;
        g.potshift = 4.0 * (1.0 / r12 - 1.0 / r6);
    }
    g.precision = p->precision;

    // Set-up, once per device, with that device current: the address of the
    // scratch array as the device sees it.  The first call on a device does
    // this (and should therefore come before any stream capture).  The address
    // is kept for the life of the process: the library must not be used on a
    // device after that device was reset (cudaDeviceReset), which unloads the
    // array and leaves the kept address stale.
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_fail(FM_ERR_NODEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 256) return na_fail(FM_ERR_NODEVICE, "device ordinal out of range");
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_na_mutex);
        if (!g_na_base[dev]) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess)
                return na_fail(FM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_na_base[dev] = static_cast<unsigned char *>(ptr);
        }
        base = g_na_base[dev];
    }
    NaScratch s = carve(base);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const int T = 256;
    k_na_zero<<<(g.ncell + T - 1) / T, T, 0, st>>>(g, s);
    k_na_bin<<<(n + T - 1) / T, T, 0, st>>>(g, s, d_r);
    k_na_scan<<<1, NA_SCAN, 0, st>>>(g, s);
    k_na_scatter<<<(n + T - 1) / T, T, 0, st>>>(g, s, d_r);
    k_na_sort<<<(g.ncell + 127) / 128, 128, 0, st>>>(g, s);
    if (g.precision == 0)
        k_na_force<0><<<(n + 127) / 128, 128, 0, st>>>(g, s, d_a, d_potenergymol, d_virialmol);
    else
        k_na_force<1><<<(n + 127) / 128, 128, 0, st>>>(g, s, d_a, d_potenergymol, d_virialmol);
    e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(FM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    unsigned int status = 0;
    e = cudaMemcpyAsync(&status, s.status, sizeof status, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_fail(FM_ERR_CUDA, std::string("status read: ") + cudaGetErrorString(e));
    if (status & 1u) return na_fail(FM_ERR_ESCAPE, "a molecule lies outside the cell grid");
    return FM_OK;
}
