// sm_100a kernels of the IMC time step.  Compiled with --fmad=false (see
// storm_device.cuh).  Each kernel names the reference lines it implements.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <type_traits>

#include "storm_device.cuh"
#include "storm_internal.h"

namespace storm {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// ------------------------------------------------------------------ bank access
__device__ __forceinline__ void load_part(const Bank &b, uint32_t q, PartReg &p) {
    p.x = b.x[q]; p.y = b.y[q]; p.z = b.z[q];
    p.vx = b.vx[q]; p.vy = b.vy[q]; p.vz = b.vz[q];
    p.t = b.t[q]; p.w = b.w[q]; p.w0 = b.w0[q];
    p.cell = b.cell[q];
    p.nu = b.nu ? b.nu[q] : 0.0;
}
__device__ __forceinline__ void store_part(const Bank &b, uint32_t q, const PartReg &p, uint32_t pid, uint32_t draw) {
    b.x[q] = p.x; b.y[q] = p.y; b.z[q] = p.z;
    b.vx[q] = p.vx; b.vy[q] = p.vy; b.vz[q] = p.vz;
    b.t[q] = p.t; b.w[q] = p.w; b.w0[q] = p.w0;
    b.cell[q] = p.cell; b.pid[q] = pid; b.draw[q] = draw;
    if (b.nu) b.nu[q] = p.nu;
}

// FP32-tracking banks reuse the same buffers: x,y,z hold the cell-local
// offsets and vx,vy,vz the direction, as floats in the first half of each buffer.
__device__ __forceinline__ void load32(const Bank &b, uint32_t q, Track32 &T) {
    T.qx = reinterpret_cast<const float *>(b.x)[q];
    T.qy = reinterpret_cast<const float *>(b.y)[q];
    T.qz = reinterpret_cast<const float *>(b.z)[q];
    T.ux = reinterpret_cast<const float *>(b.vx)[q];
    T.uy = reinterpret_cast<const float *>(b.vy)[q];
    T.uz = reinterpret_cast<const float *>(b.vz)[q];
    T.t = b.t[q]; T.w = b.w[q]; T.w0 = b.w0[q];
    T.cell = b.cell[q];
}
__device__ __forceinline__ void store32(const Bank &b, uint32_t q, const Track32 &T, uint32_t pid, uint32_t draw) {
    reinterpret_cast<float *>(b.x)[q] = T.qx;
    reinterpret_cast<float *>(b.y)[q] = T.qy;
    reinterpret_cast<float *>(b.z)[q] = T.qz;
    reinterpret_cast<float *>(b.vx)[q] = T.ux;
    reinterpret_cast<float *>(b.vy)[q] = T.uy;
    reinterpret_cast<float *>(b.vz)[q] = T.uz;
    b.t[q] = T.t; b.w[q] = T.w; b.w0[q] = T.w0;
    b.cell[q] = T.cell; b.pid[q] = pid; b.draw[q] = draw;
}
// multigroup FP32 banks keep the frequency as a float in the first half of nu
__device__ __forceinline__ float load_nu32(const Bank &b, uint32_t q) { return reinterpret_cast<const float *>(b.nu)[q]; }
__device__ __forceinline__ void store_nu32(const Bank &b, uint32_t q, float nu) { reinterpret_cast<float *>(b.nu)[q] = nu; }
// global FP64 particle -> FP32-tracking particle of its cell.  Offsets are held
// ENTRY32 of the half width inside the cell, as on a cell change: a packet
// born on a face (boundary sources) then starts a few ulps inside it, where
// the FP64 form resolves its first sub-ulp flights.
__device__ __forceinline__ void to_local(const Ctx &C, const PartReg &p, Track32 &T) {
    cell_ijk(C, p.cell, T.i, T.j, T.k);
    T.cell = p.cell;
    if (C.poly) {   // offset from the mesh point, nudged toward it
        T.qx = static_cast<float>(p.x - C.mpx[p.cell]) * ENTRY32;
        T.qy = static_cast<float>(p.y - C.mpy[p.cell]) * ENTRY32;
        T.qz = static_cast<float>(p.z - C.mpz[p.cell]) * ENTRY32;
    } else {
        T.qx = clampf(static_cast<float>(p.x - C.xc[T.i]), C.hx[T.i] * ENTRY32);
        T.qy = clampf(static_cast<float>(p.y - C.yc[T.j]), C.hy[T.j] * ENTRY32);
        T.qz = clampf(static_cast<float>(p.z - C.zc[T.k]), C.hz[T.k] * ENTRY32);
    }
    const double sp = vnorm(p.vx, p.vy, p.vz);
    const double inv = sp > 0.0 ? 1.0 / sp : 0.0;
    T.ux = static_cast<float>(p.vx * inv); T.uy = static_cast<float>(p.vy * inv); T.uz = static_cast<float>(p.vz * inv);
    T.t = p.t; T.w = p.w; T.w0 = p.w0;
    T.nu = static_cast<float>(p.nu);
}
__device__ __forceinline__ void to_global(const Ctx &C, const Track32 &T, PartReg &p) {
    uint32_t i, j, k;
    cell_ijk(C, T.cell, i, j, k);
    const double mx = C.poly ? C.mpx[T.cell] : C.xc[i], my = C.poly ? C.mpy[T.cell] : C.yc[j],
                 mz = C.poly ? C.mpz[T.cell] : C.zc[k];
    p.x = mx + static_cast<double>(T.qx);
    p.y = my + static_cast<double>(T.qy);
    p.z = mz + static_cast<double>(T.qz);
    p.vx = static_cast<double>(T.ux) * C.clight;
    p.vy = static_cast<double>(T.uy) * C.clight;
    p.vz = static_cast<double>(T.uz) * C.clight;
    p.t = T.t; p.w = T.w; p.w0 = T.w0; p.cell = T.cell;
    p.nu = static_cast<double>(T.nu);
}
// store an FP64 particle in the bank's layout
__device__ __forceinline__ void store_any(const Ctx &C, const Bank &b, uint32_t q, const PartReg &p, uint32_t pid,
                                          uint32_t draw) {
    if (C.fp32) {
        Track32 T;
        to_local(C, p, T);
        store32(b, q, T, pid, draw);
        if (b.nu) store_nu32(b, q, T.nu);
    } else {
        store_part(b, q, p, pid, draw);
    }
}
// copy one particle between banks of the same layout
__device__ __forceinline__ void copy_any(const Ctx &C, const Bank &src, uint32_t qs, const Bank &dst, uint32_t qd,
                                         uint32_t pid, uint32_t draw) {
    if (C.fp32) {
        Track32 T;
        load32(src, qs, T);
        store32(dst, qd, T, pid, draw);
    } else {
        PartReg p;
        load_part(src, qs, p);
        store_part(dst, qd, p, pid, draw);
    }
}

// ---- census bank: array of records, gathered in random order by the comb.
// FP64 form, 96 B: (x,y) (z,vx) (vy,vz) (t,w) (w0,[cell,pid]) ([draw,-],nu)
// FP32 form, 64 B: (qx,qy,qz,ux) (uy,uz,t) (w,w0) (cell,pid,draw,-)
__device__ __forceinline__ uint4 two_doubles(double a, double b) {
    const unsigned long long x = __double_as_longlong(a), y = __double_as_longlong(b);
    return make_uint4(static_cast<uint32_t>(x), static_cast<uint32_t>(x >> 32), static_cast<uint32_t>(y),
                      static_cast<uint32_t>(y >> 32));
}
__device__ __forceinline__ double lo_double(const uint4 &v) {
    return __longlong_as_double((static_cast<unsigned long long>(v.y) << 32) | v.x);
}
__device__ __forceinline__ double hi_double(const uint4 &v) {
    return __longlong_as_double((static_cast<unsigned long long>(v.w) << 32) | v.z);
}
__device__ __forceinline__ void census_store64(const CensusBank &c, uint32_t q, const PartReg &p, uint32_t pid,
                                               uint32_t draw) {
    uint4 *r = c.rec + static_cast<size_t>(q) * 6;
    r[0] = two_doubles(p.x, p.y);
    r[1] = two_doubles(p.z, p.vx);
    r[2] = two_doubles(p.vy, p.vz);
    r[3] = two_doubles(p.t, p.w);
    const unsigned long long w0 = __double_as_longlong(p.w0);
    r[4] = make_uint4(static_cast<uint32_t>(w0), static_cast<uint32_t>(w0 >> 32), p.cell, pid);
    const unsigned long long nu = __double_as_longlong(p.nu);
    r[5] = make_uint4(draw, 0u, static_cast<uint32_t>(nu), static_cast<uint32_t>(nu >> 32));
}
__device__ __forceinline__ void census_load64(const CensusBank &c, uint32_t q, PartReg &p, uint32_t &pid,
                                              uint32_t &draw) {
    const uint4 *r = c.rec + static_cast<size_t>(q) * 6;
    const uint4 a = r[0], b = r[1], d = r[2], e = r[3], f = r[4], g = r[5];
    p.x = lo_double(a); p.y = hi_double(a);
    p.z = lo_double(b); p.vx = hi_double(b);
    p.vy = lo_double(d); p.vz = hi_double(d);
    p.t = lo_double(e); p.w = hi_double(e);
    p.w0 = lo_double(f);
    p.cell = f.z; pid = f.w; draw = g.x;
    p.nu = hi_double(g);
}
__device__ __forceinline__ void census_store32(const CensusBank &c, uint32_t q, const Track32 &T, uint32_t pid,
                                               uint32_t draw) {
    uint4 *r = c.rec + static_cast<size_t>(q) * 4;
    r[0] = make_uint4(__float_as_uint(T.qx), __float_as_uint(T.qy), __float_as_uint(T.qz), __float_as_uint(T.ux));
    const unsigned long long t = __double_as_longlong(T.t);
    r[1] = make_uint4(__float_as_uint(T.uy), __float_as_uint(T.uz), static_cast<uint32_t>(t), static_cast<uint32_t>(t >> 32));
    r[2] = two_doubles(T.w, T.w0);
    r[3] = make_uint4(T.cell, pid, draw, 0u);
}
// the same record with the frequency (multigroup) in its last word
__device__ __forceinline__ void census_store32_mg(const CensusBank &c, uint32_t q, const Track32 &T, uint32_t pid,
                                                  uint32_t draw) {
    census_store32(c, q, T, pid, draw);
    reinterpret_cast<uint32_t *>(c.rec + static_cast<size_t>(q) * 4 + 3)[3] = __float_as_uint(T.nu);
}
__device__ __forceinline__ void census_load32(const CensusBank &c, uint32_t q, Track32 &T, uint32_t &pid,
                                              uint32_t &draw) {
    const uint4 *r = c.rec + static_cast<size_t>(q) * 4;
    const uint4 a = r[0], b = r[1], d = r[2], e = r[3];
    T.qx = __uint_as_float(a.x); T.qy = __uint_as_float(a.y); T.qz = __uint_as_float(a.z); T.ux = __uint_as_float(a.w);
    T.uy = __uint_as_float(b.x); T.uz = __uint_as_float(b.y);
    T.t = __longlong_as_double((static_cast<unsigned long long>(b.w) << 32) | b.z);
    T.w = lo_double(d); T.w0 = hi_double(d);
    T.cell = e.x; pid = e.y; draw = e.z;
    T.nu = __uint_as_float(e.w);
}
// weight, cell and pid of census record q
__device__ __forceinline__ double census_w(const Ctx &C, const CensusBank &c, uint32_t q) {
    const uint4 v = c.rec[static_cast<size_t>(q) * (C.fp32 ? 4 : 6) + (C.fp32 ? 2 : 3)];
    return C.fp32 ? lo_double(v) : hi_double(v);
}
__device__ __forceinline__ uint2 census_cell_pid(const Ctx &C, const CensusBank &c, uint32_t q) {
    const uint4 v = c.rec[static_cast<size_t>(q) * (C.fp32 ? 4 : 6) + (C.fp32 ? 3 : 4)];
    return C.fp32 ? make_uint2(v.x, v.y) : make_uint2(v.z, v.w);
}

// convert a bank between the FP64 (global) and FP32-tracking (local) layouts
__global__ void k_bank_to_local(Ctx C, Bank src, Bank dst, uint32_t lo, uint32_t n) {
    for (uint32_t q = lo + blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        PartReg p;
        load_part(src, q, p);
        Track32 T;
        to_local(C, p, T);
        store32(dst, q, T, src.pid[q], src.draw[q]);
        if (dst.nu) store_nu32(dst, q, T.nu);
    }
}
__global__ void k_bank_to_census(Ctx C, Bank src, CensusBank dst, uint32_t n) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        PartReg p;
        load_part(src, q, p);
        if (C.fp32) {
            Track32 T;
            to_local(C, p, T);
            if (C.groups >= 2) census_store32_mg(dst, q, T, src.pid[q], src.draw[q]);
            else census_store32(dst, q, T, src.pid[q], src.draw[q]);
        } else {
            census_store64(dst, q, p, src.pid[q], src.draw[q]);
        }
    }
}
__global__ void k_bank_to_global(Ctx C, Bank src, Bank dst, uint32_t n) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        Track32 T;
        load32(src, q, T);
        T.nu = src.nu ? load_nu32(src, q) : 0.0f;
        PartReg p;
        to_global(C, T, p);
        store_part(dst, q, p, src.pid[q], src.draw[q]);
    }
}

// ------------------------------------------------------------------ step start
// manager step() (manager/MonteCarloManagerSerial.hpp:393-405): census particles
// get timeLeft = dt, initialWeight = |w|; they take pids pidOffset + 0..n-1
// (pidOffset: the census of the shards below this handle's, 0 unsharded).
__global__ void k_begin(Bank b, uint32_t lo, uint32_t n, uint32_t pidOffset, double dt, DevStats *st) {
    double e = 0.0;
    for (uint32_t q = lo + blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        double w = b.w[q];
        b.t[q] = dt;
        b.w0[q] = fabs(w);
        b.pid[q] = pidOffset + q;
        b.draw[q] = 0;
        e += w;
    }
    e = warp_sum(e);
    if ((threadIdx.x & 31) == 0 && e != 0.0) atomicAdd(&st->eCensusIn, e);
}

// mean chord 4V/S of a cell (computeCellSurfaceArea, radiation/RadiationIMC.hpp:971-980, GetCellFaces order)
__device__ __forceinline__ double cell_chord(const Ctx &C, const CellArrays &A, uint32_t c) {
    if (C.poly) return C.chord[c];   // 4 V / S with S summed in GetCellFaces order on the host
    uint32_t i, j, k;
    cell_ijk(C, c, i, j, k);
    double dx = C.xe[i + 1] - C.xe[i], dy = C.ye[j + 1] - C.ye[j], dz = C.ze[k + 1] - C.ze[k];
    double ax = dy * dz, ay = dz * dx, az = dx * dy;
    double S = 0.0;
    S += ax; S += ax; S += ay; S += ay; S += az; S += az;
    return (S > 0.0) ? 4.0 * A.vol[c] / S : 0.0;
}

// Random Walk eligibility of a cell (precomputeRandomWalkData, radiation/RadiationIMC.hpp:982-1063,
// with computeCellSurfaceArea :971-980 in GetCellFaces order) and the FP32
// form's segment constants: x = 1/sigma_e (inf when none), y = sigma_a f,
// z = rwMinParticleOpticalDepth / sigma_T, the distance to the nearest face a
// particle needs for a Random Walk jump (inf in cells that are not eligible),
// w = -1 / (sigma_a f c), the factor from exp-deposit to time-integrated energy.
__device__ __forceinline__ void cell_rw_and_phys32(const Ctx &C, const CellArrays &A, uint32_t c, double sa, double ss,
                                                   double f) {
    const double sigmaT = sa + ss;
    bool elig = false;
    if (C.withRW) {
        if (C.groups >= 2) {   // PGRW: eligible where some groups are diffusive (tables from prestep)
            elig = A.pgrwCut[c] > 0;
            A.rwSigT[c] = elig ? A.pgrw[c].x : sigmaT;
        } else {
            A.rwSigT[c] = sigmaT;
            elig = sigmaT * cell_chord(C, A, c) >= C.rwMinCell;
        }
        A.rwElig[c] = elig ? 1 : 0;
    }
    if (C.fp32 && C.groups >= 2) {
        // multigroup: x = elastic opacity, y = Fleck factor, z = PGRW reach, w = PGRW D
        const double4 g4 = A.pgrw[c];
        const bool rw = elig && g4.x > 0.0;
        A.phys32[c] = make_float4(static_cast<float>(ss), static_cast<float>(f),
                                  rw ? static_cast<float>(C.rwMinParticle / g4.x) : CUDART_INF_F,
                                  rw ? static_cast<float>(g4.z) : 0.0f);
    } else if (C.fp32) {
        const double eventOpacity = ss + (1.0 - f) * sa;
        const bool rw = elig && sigmaT > 0.0;
        const double rate = sa * f * C.clight;
        A.phys32[c] = make_float4(eventOpacity > 0.0 ? static_cast<float>(1.0 / eventOpacity) : CUDART_INF_F,
                                  static_cast<float>(sa * f),
                                  rw ? static_cast<float>(C.rwMinParticle / sigmaT) : CUDART_INF_F,
                                  rate > 0.0 ? static_cast<float>(-1.0 / rate) : 0.0f);
    }
}

// ------------------------------------------------------------------ prestep
// RadiationIMC::preStep (radiation/RadiationIMC.hpp:1618-1661) per cell, the opacity
// plug-in (CalcPlanckOpacity / CalcScatteringOpacity) and precomputeRandomWalkData
// (:982-1006, gray branch); clears Erad_time_avg_.
// Multigroup per-cell tables: the Planck mean opacity of the opacity plug-in
// (examples/densmore2012/DensmoreOpacity.hpp:36-56), the cumulative emission
// spectrum sum_g sigma_g B_g it samples from (:146-165), and the PGRW data of
// precomputeRandomWalkData (radiation/RadiationIMC.hpp:1008-1061).  Every
// group weight is evaluated at the group centre with planck_integral.
__device__ inline double mg_cell_tables(const Ctx &C, const CellArrays &A, uint32_t c, double scat, double chord) {
    const uint32_t G = C.groups;
    const double T = C.T[c];
    const double kT = C.kBoltz * (T < 1.0 ? 1.0 : T);   // the opacity model's kT
    const double kTrw = C.kBoltz * T;                    // precomputeRandomWalkData's kT
    double *cdf = A.mgCdf + static_cast<size_t>(c) * (G + 1);
    double weightedSum = 0.0, totalWeight = 0.0, cum = 0.0;
    double totalSigABgAll = 0.0, totalBgDiff = 0.0, sumBgSigADiff = 0.0, sumBgSigTDiff = 0.0, sumBgOverSigTDiff = 0.0;
    uint32_t cutoff = 0;
    bool foundNonDiffusive = false;
    cdf[0] = 0.0;
    const double kTq = pow(kT, C.mgQ);   // the same in every group
    C.mgKTq[c] = kTq;
    PiBound lo = pi_bound(C.gb[0] / kT);
    for (uint32_t g = 0; g < G; ++g) {
        const double b0 = C.gb[g], b1 = C.gb[g + 1];
        const double Ec = 0.5 * (b0 + b1);
        const PiBound hi = pi_bound(b1 / kT);
        const double a = lo.x, b = hi.x;   // b0 / kT, b1 / kT
        const double Bg = (a > 0.0 && b > a) ? pi_between(lo, hi) : 0.0;
        lo = hi;
        const double sg = mg_sigma(C, c, Ec, kT, kTq, C.mgEp[g]);   // = CalcAbsorptionOpacity(cell, centre of g)
        weightedSum += sg * Bg;
        totalWeight += Bg;
        const double weight = (sg > 0.0 && isfinite(sg) && isfinite(Bg)) ? sg * Bg : 0.0;
        cum = cum + weight;
        cdf[g + 1] = cum;
        if (C.withRW) {
            double Bgr;
            if (kTrw == kT) {
                Bgr = (a > 0.0 && b > a) ? Bg : 1.0 / static_cast<double>(G);
            } else {
                const double ar = b0 / kTrw, br = b1 / kTrw;
                Bgr = (ar > 0.0 && br > ar) ? planck_integral(ar, br) : 1.0 / static_cast<double>(G);
            }
            const double sigT = sg + scat;
            totalSigABgAll += sg * Bgr;
            if (!foundNonDiffusive && sigT * chord >= C.rwMinCell) {
                cutoff = g + 1;
                totalBgDiff += Bgr;
                sumBgSigADiff += Bgr * sg;
                sumBgSigTDiff += Bgr * sigT;
                if (sigT > 0.0) sumBgOverSigTDiff += Bgr / sigT;
            } else {
                foundNonDiffusive = true;
            }
        }
    }
    const double sigmaP = (totalWeight > 0.0) ? weightedSum / totalWeight : 1e-20;
    if (C.withRW) {
        if (cutoff > 0 && totalBgDiff > 0.0) {
            A.pgrwCut[c] = cutoff;
            A.pgrw[c] = make_double4(sumBgSigTDiff / totalBgDiff, sumBgSigADiff / totalBgDiff,
                                     (C.clight / 3.0) * sumBgOverSigTDiff / totalBgDiff,
                                     (totalSigABgAll > 0.0) ? sumBgSigADiff / totalSigABgAll : 1.0);
        } else {
            A.pgrwCut[c] = 0;
            A.pgrw[c] = make_double4(0.0, 0.0, 0.0, 0.0);
        }
    }
    return sigmaP;
}

// precomputeDDMCData, first loop (radiation/RadiationIMC.hpp:1283-1353): the
// cell's DDMC opacities and diffusion coefficient.  Gray (and multigroup without
// ddmcUseMultigroupPGRW): sigma_A = the Planck opacity, sigma_T = sigma_A +
// sigma_s, D = c / (3 sigma_T), eligible where sigma_T 4V/S >= the cell depth.
// The multigroup PGRW form averages the diffusive groups (those below the first
// group with sigma_T,g 4V/S under the cell depth) with equal weights 1/G.
__device__ inline void ddmc_cell_data(const Ctx &C, const CellArrays &A, uint32_t c, double sa, double ss) {
    const double chord = cell_chord(C, A, c);
    double sigmaA = 0.0, sigmaT = 0.0, D = 0.0, eligible = 0.0;
    uint32_t cutoff = 0;
    if (chord > 0.0) {
        if (C.ddmcPgrw) {
            const double T = C.T[c];
            if (C.kBoltz * T > 0.0) {
                const uint32_t G = C.groups;
                const double kT = mg_kT(C, c);
                const double kTq = C.mgKTq[c];
                const double Bg = 1.0 / static_cast<double>(G);
                double totalBgDiff = 0.0, sumA = 0.0, sumT = 0.0, sumOver = 0.0;
                bool foundNonDiffusive = false;
                for (uint32_t g = 0; g < G; ++g) {
                    const double Ec = 0.5 * (C.gb[g] + C.gb[g + 1]);
                    const double sigA = mg_sigma(C, c, Ec, kT, kTq, C.mgEp[g]);
                    const double sigT = sigA + ss;
                    if (!foundNonDiffusive && sigT * chord >= C.ddmcMinCell) {
                        cutoff = g + 1;
                        totalBgDiff += Bg;
                        sumA += Bg * sigA;
                        sumT += Bg * sigT;
                        if (sigT > 0.0) sumOver += Bg / sigT;
                    } else {
                        foundNonDiffusive = true;
                    }
                }
                if (cutoff > 0 && totalBgDiff > 0.0) {
                    sigmaA = sumA / totalBgDiff;
                    sigmaT = sumT / totalBgDiff;
                    D = (C.clight / 3.0) * sumOver / totalBgDiff;
                    eligible = (sigmaT > 0.0 && D > 0.0) ? 1.0 : 0.0;
                } else {
                    cutoff = 0;
                }
            }
        } else {
            sigmaA = sa;
            sigmaT = sigmaA + ss;
            D = (sigmaT > 0.0) ? C.clight / (3.0 * sigmaT) : 0.0;
            eligible = (sigmaT * chord >= C.ddmcMinCell && D > 0.0) ? 1.0 : 0.0;
        }
    }
    C.ddmc[c] = make_double4(sigmaT, sigmaA, eligible, D);
    if (C.ddmcCut) C.ddmcCut[c] = cutoff;
}

__global__ void k_prestep(Ctx C, CellArrays A, OpacityEos M, double dt) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        double sa, ss;
        const double T = A.T[c];
        if (C.groups >= 2) {
            ss = M.tabS ? M.tabS[c] : 0.0;
            sa = mg_cell_tables(C, A, c, ss, C.withRW ? cell_chord(C, A, c) : 0.0);
        } else if (M.opacityKind == STORM_OPACITY_CELL_TABLE) {
            sa = M.tabA[c];
            ss = M.tabS ? M.tabS[c] : 0.0;
        } else {
            double tmax = T < M.tFloor ? M.tFloor : T;   // std::max(T, floor)
            double tf = pow(C.kevKelvin / tmax, M.alpha);
            double rf = M.rhoF ? M.rhoF[c] : 1.0;
            double kk = M.kP0 * tf * rf;
            sa = (M.cap > 0.0) ? (M.cap < kk ? M.cap : kk) : kk;
            if (M.kR0 > 0.0) {
                double kR = M.kR0 * tf * rf, kP = M.kP0 * tf * rf;
                double sd = kR - kP;
                ss = sd > 0.0 ? sd : 0.0;   // std::max(kR - kP, 0)
            } else {
                ss = 0.0;
            }
        }
        A.sigA[c] = sa;
        A.sigS[c] = ss;
        A.eradAvg[c] = 0.0;
        double cv;
        if (M.eosKind == STORM_EOS_LINEAR) {
            cv = M.cvPerMass;
        } else {
            double rho = A.mass[c] / A.vol[c];
            double Tm = T < 1.0 ? 1.0 : T;
            cv = M.eosF * M.eosBeta * pow(Tm, M.eosBeta - 1.0) * pow(rho, 1.0 - M.eosMu) / rho;
        }
        double T3 = (T * T) * T;   // boost::math::pow<3>
        double gamma = 1.0;        // moving material: the cell's Lorentz factor (:1636-1644)
        if (C.withHydro) {
            double4 v = C.vel[c];
            gamma = 1.0 / sqrt(1.0 - ((v.x * v.x + v.y * v.y) + v.z * v.z) * C.invC2);
            v.w = gamma;
            C.vel[c] = v;
        }
        double f = 1.0 / (1.0 + (4.0 * C.arad * T3 * sa * C.clight * dt * gamma) / cv);
        A.fleck[c] = f;
        if (f < 0.0 || f > 1.0) raise_error(C, STORM_DERR_FLECK, c, 0);
        A.phys[c] = cell_phys(sa, ss, f, sa + ss, C.clight);
        cell_rw_and_phys32(C, A, c, sa, ss, f);
        if (C.withDDMC) ddmc_cell_data(C, A, c, sa, ss);
    }
}

// precomputeDDMCData, second loop (radiation/RadiationIMC.hpp:1355-1413): the
// leak rate through each face to a neighbour inside the box,
// D_face A / (V d) with D_face the harmonic mean of the two cells' D (the
// cell's own D where the neighbour has none) and d the distance from the cell
// centre to the face; cells whose rates sum to zero are not eligible.  The
// FP32 form's per-cell copy holds the particle depth it needs, 1/total, the
// absorption rate sigma_A f c, the PGRW frequency bound and the cumulative
// face fractions.
// precomputeDDMCData's second loop on a convex-polyhedral cell
// (radiation/RadiationIMC.hpp:1355-1413): per cell-face slot, GetCellFaces
// order, faces on the box excluded; the face distance from the face centroid
// along the unit normal (the inward slot normal, the same up to its sign), or
// half the distance to the neighbour's mesh point where that is zero.  The
// FP32 form's header holds what the Cartesian one holds, with the last slot
// that has a rate; the cumulative face fractions go per slot.
__device__ inline void ddmc_rates_poly(const Ctx &C, const CellArrays &A, uint32_t c, const double4 &dd) {
    const uint32_t k0 = C.cfo[c], k1 = C.cfo[c + 1];
    double total = 0.0;
    if (dd.z > 0.0) {
        const double volume = A.vol[c];
        const double D1 = dd.w;
        const double mx = C.mpx[c], my = C.mpy[c], mz = C.mpz[c];
        for (uint32_t k = k0; k < k1; ++k) {
            double rate = 0.0;
            const uint32_t nb = C.cfNext[k];
            if (nb < C.ncells) {
                const double4 n = C.cfN[k], q = C.cfP[k];
                double faceDistance = fabs((q.x - mx) * n.x + (q.y - my) * n.y + (q.z - mz) * n.z);
                if (!(faceDistance > 0.0))
                    faceDistance = 0.5 * fabs((C.mpx[nb] - mx) * n.x + (C.mpy[nb] - my) * n.y + (C.mpz[nb] - mz) * n.z);
                if (faceDistance > 0.0) {
                    double diffusionFace = D1;
                    const double D2 = C.ddmc[nb].w;
                    if (D2 > 0.0)
                        diffusionFace = (D1 > 0.0 && D2 > 0.0) ? (2.0 * D1 * D2 / (D1 + D2)) : (D1 < D2 ? D2 : D1);
                    const double r = diffusionFace * C.cfA[k] / (volume * faceDistance);
                    if (r > 0.0 && isfinite(r)) rate = r;
                }
            }
            C.ddmcRate[k] = rate;
            total += rate;
        }
    }
    if (!(total > 0.0)) {
        total = 0.0;
        for (uint32_t k = k0; k < k1; ++k) C.ddmcRate[k] = 0.0;
    }
    C.ddmcTot[c] = total;
    if (C.fp32) {
        float4 *o32 = C.ddmc32 + static_cast<size_t>(c) * 3;
        if (total > 0.0) {
            double acc = 0.0;
            int last = -1;
            for (uint32_t k = k0; k < k1; ++k) {
                acc += C.ddmcRate[k];
                C.ddmcCum32[k] = static_cast<float>(acc / total);
                if (C.ddmcRate[k] > 0.0) last = static_cast<int>(k - k0);
            }
            o32[0] = make_float4(static_cast<float>(C.ddmcMinParticle / dd.x), static_cast<float>(1.0 / total),
                                 static_cast<float>(dd.y * A.fleck[c] * C.clight), CUDART_INF_F);
            o32[1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            o32[2] = make_float4(0.0f, 0.0f, static_cast<float>(last), 0.0f);
        } else {
            o32[0] = make_float4(CUDART_INF_F, 0.0f, 0.0f, 0.0f);
            o32[1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            o32[2] = make_float4(0.0f, 0.0f, -1.0f, 0.0f);
        }
    }
}

__global__ void k_ddmc_rates(Ctx C, CellArrays A) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        const double4 dd = C.ddmc[c];
        if (C.poly) {
            ddmc_rates_poly(C, A, c, dd);
            continue;
        }
        double rates[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        double total = 0.0;
        uint32_t i, j, k;
        cell_ijk(C, c, i, j, k);
        if (dd.z > 0.0) {
            const double dx = C.xe[i + 1] - C.xe[i], dy = C.ye[j + 1] - C.ye[j], dz = C.ze[k + 1] - C.ze[k];
            const double volume = (dx * dy) * dz;
            const double D1 = dd.w;
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                uint32_t next;
                bool inside;
                double faceDistance, area;
                switch (s) {
                case 0: inside = i > 0; next = c - 1; faceDistance = fabs(C.xe[i] - C.xc[i]); area = dy * dz; break;
                case 1: inside = i + 1 < C.nx; next = c + 1; faceDistance = fabs(C.xe[i + 1] - C.xc[i]); area = dy * dz; break;
                case 2: inside = j > 0; next = c - C.nx; faceDistance = fabs(C.ye[j] - C.yc[j]); area = dz * dx; break;
                case 3: inside = j + 1 < C.ny; next = c + C.nx; faceDistance = fabs(C.ye[j + 1] - C.yc[j]); area = dz * dx; break;
                case 4: inside = k > 0; next = c - C.nx * C.ny; faceDistance = fabs(C.ze[k] - C.zc[k]); area = dx * dy; break;
                default: inside = k + 1 < C.nz; next = c + C.nx * C.ny; faceDistance = fabs(C.ze[k + 1] - C.zc[k]); area = dx * dy; break;
                }
                if (!inside || !(faceDistance > 0.0)) continue;
                double diffusionFace = D1;
                const double D2 = C.ddmc[next].w;
                if (D2 > 0.0) diffusionFace = (D1 > 0.0 && D2 > 0.0) ? (2.0 * D1 * D2 / (D1 + D2)) : (D1 < D2 ? D2 : D1);
                const double rate = diffusionFace * area / (volume * faceDistance);
                if (rate > 0.0 && isfinite(rate)) {
                    rates[s] = rate;
                    total += rate;
                }
            }
            if (!(total > 0.0)) {
                total = 0.0;
                for (int s = 0; s < 6; ++s) rates[s] = 0.0;
            }
        }
        C.ddmcTot[c] = total;
        double *out = C.ddmcRate + static_cast<size_t>(c) * 6;
        for (int s = 0; s < 6; ++s) out[s] = rates[s];
        if (C.fp32) {
            float4 *o32 = C.ddmc32 + static_cast<size_t>(c) * 3;
            if (total > 0.0) {
                float bound = CUDART_INF_F;
                float reach = static_cast<float>(C.ddmcMinParticle / dd.x);
                if (C.ddmcPgrw) {
                    const uint32_t cut = C.ddmcCut[c];
                    if (cut == 0 || cut > C.groups) reach = CUDART_INF_F;
                    else bound = C.gb32[cut];
                }
                float cum[6];
                double acc = 0.0;
                int last = -1;
                for (int s = 0; s < 6; ++s) {
                    acc += rates[s];
                    cum[s] = static_cast<float>(acc / total);
                    if (rates[s] > 0.0) last = s;
                }
                o32[0] = make_float4(reach, static_cast<float>(1.0 / total),
                                     static_cast<float>(dd.y * A.fleck[c] * C.clight), bound);
                o32[1] = make_float4(cum[0], cum[1], cum[2], cum[3]);
                o32[2] = make_float4(cum[4], cum[5], static_cast<float>(last), 0.0f);
            } else {
                o32[0] = make_float4(CUDART_INF_F, 0.0f, 0.0f, 0.0f);
                o32[1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                o32[2] = make_float4(0.0f, 0.0f, -1.0f, 0.0f);
            }
        }
    }
}

// Segment constants and RW eligibility from externally supplied tables
// (storm_cuda_set_cell_physics).
__global__ void k_rw_eligibility(Ctx C, CellArrays A) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        double sigmaT = A.sigA[c] + A.sigS[c];
        A.phys[c] = cell_phys(A.sigA[c], A.sigS[c], A.fleck[c], sigmaT, C.clight);
        cell_rw_and_phys32(C, A, c, A.sigA[c], A.sigS[c], A.fleck[c]);
    }
}

// ------------------------------------------------------------------ emission allocation
// generateParticles (radiation/RadiationIMC.hpp:2047-2059): energy per cell.
__global__ void k_emission_energy(Ctx C, CellArrays A, double dt) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        double T = A.T[c];
        double T4 = (T * T) * (T * T);   // boost::math::pow<4>
        A.emitE[c] = A.fleck[c] * A.vol[c] * C.arad * T4 * A.sigA[c] * dt * C.clight;
    }
}

// localTotalEnergy += energyToCreateVec[i] (:2058-2059) in the reference's order:
// one thread adds the cells left to right so the allocation below floors against
// the same total, bit for bit.  A warp streams the values through shared memory.
// onlyIf: when not null, the kernel runs only if *onlyIf is nonzero (a device-side
// fallback that needs no host readback).
__global__ void k_sequential_sum(const double *v, uint32_t n, double *out, const int32_t *onlyIf) {
    if (onlyIf && *onlyIf == 0) return;
    __shared__ double buf[1024];
    double s = 0.0;
    for (uint32_t base = 0; base < n; base += 1024) {
        for (uint32_t q = threadIdx.x; q < 1024 && base + q < n; q += blockDim.x) buf[q] = v[base + q];
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t m = (n - base) < 1024 ? (n - base) : 1024;
            for (uint32_t q = 0; q < m; ++q) s += buf[q];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s;
}

// nPhotonsVec (:2071-2087)
__global__ void k_allocate(Ctx C, CellArrays A, const double *total, uint64_t newPerCell, const int32_t *onlyIf) {
    if (onlyIf && *onlyIf == 0) return;
    const double tot = *total;
    const uint64_t totalParticles = static_cast<uint64_t>(C.ncells) * newPerCell * 10;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        double E = A.emitE[c];
        uint64_t share = (tot > 0) ? static_cast<uint64_t>(E / tot * static_cast<double>(totalParticles)) : newPerCell;
        uint64_t cap = newPerCell * 20;
        uint64_t m = share < cap ? share : cap;
        A.photons[c] = (E > 0.0) ? (m > newPerCell ? m : newPerCell) : 0;
    }
}

// The same counts from a fast deterministic total.  E_i >= 0, so the reference's
// left-to-right total and this blocked total both lie within rel * total of the
// exact sum (rel bounds the rounding of either order).  floor(fl(fl(E/S) * T)) is
// monotone in S, so when it agrees at both ends of that interval it equals the
// count the reference's total gives; otherwise the cell is flagged and the
// caller recomputes everything with the exact sequential total.
__global__ void k_allocate_checked(Ctx C, CellArrays A, const double *total, uint64_t newPerCell, double rel,
                                   int32_t *ambiguous) {
    const double tot = *total;
    const uint64_t totalParticles = static_cast<uint64_t>(C.ncells) * newPerCell * 10;
    const double lo = tot * (1.0 - rel), hi = tot * (1.0 + rel);
    int amb = 0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        double E = A.emitE[c];
        uint64_t share = (tot > 0) ? static_cast<uint64_t>(E / tot * static_cast<double>(totalParticles)) : newPerCell;
        if (tot > 0 && E > 0.0) {
            uint64_t a = static_cast<uint64_t>(E / lo * static_cast<double>(totalParticles));
            uint64_t b = static_cast<uint64_t>(E / hi * static_cast<double>(totalParticles));
            if (a != b) amb = 1;
        }
        uint64_t cap = newPerCell * 20;
        uint64_t m = share < cap ? share : cap;
        A.photons[c] = (E > 0.0) ? (m > newPerCell ? m : newPerCell) : 0;
    }
    if (__any_sync(FULL, amb) && (threadIdx.x & 31) == 0) atomicOr(ambiguous, 1);
}

// material debit (:2193-2195)
__global__ void k_emission_debit(Ctx C, CellArrays A, DevStats *st) {
    double deb = 0.0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        if (A.photons[c] == 0) continue;
        double E = A.emitE[c];
        if (!C.noFeedback) A.eint[c] -= E;
        if (C.withHydro && !C.noFeedback) {   // momentum carried off by the emission (:2200-2206)
            const double4 v = C.vel[c];
            double *m = C.mom + 3 * static_cast<size_t>(c);
            m[0] -= E * v.x * C.invC2 * v.w;
            m[1] -= E * v.y * C.invC2 * v.w;
            m[2] -= E * v.z * C.invC2 * v.w;
        }
        deb += E;
    }
    deb = warp_sum(deb);
    if ((threadIdx.x & 31) == 0 && deb != 0.0) atomicAdd(&st->eDebit, deb);
}

// ------------------------------------------------------------------ exclusive scan (uint64)
// Three phases: per-block inclusive scan of 1024-element tiles, scan of the tile
// totals by one block, add-back.  Output out[0..n] with out[n] = total.
__device__ __forceinline__ uint64_t block_scan_incl(uint64_t v, uint64_t *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        uint64_t s = (lane < (blockDim.x >> 5)) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(FULL, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    if (wid > 0) v += sh[wid - 1];
    __syncthreads();
    return v;
}
__global__ void k_scan_tiles(const uint64_t *in, uint32_t n, uint64_t *out, uint64_t *tileSums) {
    __shared__ uint64_t sh[32];
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t v = q < n ? in[q] : 0;
    uint64_t inc = block_scan_incl(v, sh);
    if (q < n) out[q] = inc - v;
    if (threadIdx.x == blockDim.x - 1) tileSums[blockIdx.x] = inc;
}
__global__ void k_scan_sums(uint64_t *tileSums, uint32_t ntiles, uint64_t *total) {
    __shared__ uint64_t sh[32];
    __shared__ uint64_t last;
    uint64_t carry = 0;
    for (uint32_t base = 0; base < ntiles; base += blockDim.x) {
        uint32_t q = base + threadIdx.x;
        uint64_t v = q < ntiles ? tileSums[q] : 0;
        uint64_t inc = block_scan_incl(v, sh);
        if (q < ntiles) tileSums[q] = carry + inc - v;
        if (threadIdx.x == blockDim.x - 1) last = inc;
        __syncthreads();
        carry += last;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}
__global__ void k_scan_add(uint64_t *out, uint32_t n, const uint64_t *tileSums, const uint64_t *total) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) out[q] += tileSums[blockIdx.x];
    if (q == 0) out[n] = *total;
}

// ------------------------------------------------------------------ samplers
// Vertex coordinates of side s of cell (i,j,k) in the grid's GetPointsInFace order.
__device__ __forceinline__ void face_vertices(const Ctx &C, uint32_t i, uint32_t j, uint32_t k, int s, double q[4][3]) {
    int axis = s >> 1, hi = s & 1;
    if (axis == 0) {
        double X = C.xe[i + hi];
        double y0 = C.ye[j], y1 = C.ye[j + 1], z0 = C.ze[k], z1 = C.ze[k + 1];
        q[0][0] = X; q[0][1] = y0; q[0][2] = z0;
        q[1][0] = X; q[1][1] = y1; q[1][2] = z0;
        q[2][0] = X; q[2][1] = y1; q[2][2] = z1;
        q[3][0] = X; q[3][1] = y0; q[3][2] = z1;
    } else if (axis == 1) {
        double Y = C.ye[j + hi];
        double x0 = C.xe[i], x1 = C.xe[i + 1], z0 = C.ze[k], z1 = C.ze[k + 1];
        q[0][0] = x0; q[0][1] = Y; q[0][2] = z0;
        q[1][0] = x0; q[1][1] = Y; q[1][2] = z1;
        q[2][0] = x1; q[2][1] = Y; q[2][2] = z1;
        q[3][0] = x1; q[3][1] = Y; q[3][2] = z0;
    } else {
        double Z = C.ze[k + hi];
        double x0 = C.xe[i], x1 = C.xe[i + 1], y0 = C.ye[j], y1 = C.ye[j + 1];
        q[0][0] = x0; q[0][1] = y0; q[0][2] = Z;
        q[1][0] = x1; q[1][1] = y0; q[1][2] = Z;
        q[2][0] = x1; q[2][1] = y1; q[2][2] = Z;
        q[3][0] = x0; q[3][1] = y1; q[3][2] = Z;
    }
}

// RandomInCellPositionSampler::operator() (utils/RandomInCell.hpp:11-67): pick one
// of the 12 fan tetrahedra by volume, then a uniform point in it.
template <class RNG>
__device__ inline void sample_in_cell(const Ctx &C, uint32_t cell, RNG &rng, double &px, double &py, double &pz) {
    uint32_t i, j, k;
    cell_ijk(C, cell, i, j, k);
    const double cx = C.xc[i], cy = C.yc[j], cz = C.zc[k];
    double cum[12];
    double total = 0.0;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        double q[4][3];
        face_vertices(C, i, j, k, s, q);
#pragma unroll
        for (int t = 1; t < 3; ++t) {
            double ax = q[0][0] - cx, ay = q[0][1] - cy, az = q[0][2] - cz;
            double bx = q[t][0] - cx, by = q[t][1] - cy, bz = q[t][2] - cz;
            double ex = q[t + 1][0] - cx, ey = q[t + 1][1] - cy, ez = q[t + 1][2] - cz;
            double crx = by * ez - bz * ey, cry = bz * ex - bx * ez, crz = bx * ey - by * ex;
            double vol = fabs(ax * crx + ay * cry + az * crz);
            total += vol;
            cum[2 * s + (t - 1)] = total;
        }
    }
    double r = rng.raw() * total;
    // std::lower_bound over the 12 cumulative volumes
    uint32_t first = 0, count = 12;
    while (count > 0) {
        uint32_t step = count >> 1, it = first + step;
        if (cum[it] < r) { first = it + 1; count -= step + 1; } else count = step;
    }
    if (first >= 12) first = 11;
    double s = rng.raw(), t = rng.raw(), u = rng.raw(), tmp;
    if (s > t) { tmp = s; s = t; t = tmp; }
    if (t > u) { tmp = t; t = u; u = tmp; }
    if (s > t) { tmp = s; s = t; t = tmp; }
    const int side = first >> 1, tri = (first & 1) + 1;
    double q[4][3];
    face_vertices(C, i, j, k, side, q);
    const double a0 = s, a1 = t - s, a2 = u - t, a3 = 1 - u;
    px = a0 * q[0][0] + a1 * q[tri][0] + a2 * q[tri + 1][0] + a3 * cx;
    py = a0 * q[0][1] + a1 * q[tri][1] + a2 * q[tri + 1][1] + a3 * cy;
    pz = a0 * q[0][2] + a1 * q[tri][2] + a2 * q[tri + 1][2] + a3 * cz;
}

// The same sampler on a convex-polyhedral cell: the fan triangles
// (v0, v_t, v_t+1) of each face polygon, faces in GetCellFaces order, make
// tetrahedra with the mesh point; one is picked by std::lower_bound over the
// running volume sum (summed again on the second pass, bit for bit), then the
// point from three sorted uniforms.
__device__ __forceinline__ double poly_tet_volume(const Ctx &C, uint32_t v0, uint32_t v1, uint32_t v2, double cx,
                                                  double cy, double cz) {
    const double ax = C.vtx[3 * v0] - cx, ay = C.vtx[3 * v0 + 1] - cy, az = C.vtx[3 * v0 + 2] - cz;
    const double bx = C.vtx[3 * v1] - cx, by = C.vtx[3 * v1 + 1] - cy, bz = C.vtx[3 * v1 + 2] - cz;
    const double ex = C.vtx[3 * v2] - cx, ey = C.vtx[3 * v2 + 1] - cy, ez = C.vtx[3 * v2 + 2] - cz;
    const double crx = by * ez - bz * ey, cry = bz * ex - bx * ez, crz = bx * ey - by * ex;
    return fabs(ax * crx + ay * cry + az * crz);
}
template <class RNG>
__device__ inline void sample_in_poly_cell(const Ctx &C, uint32_t cell, RNG &rng, double &px, double &py, double &pz) {
    const double cx = C.mpx[cell], cy = C.mpy[cell], cz = C.mpz[cell];
    uint32_t v0 = 0, v1 = 0, v2 = 0;
    if (C.tetCum) {
        // the running sums of the mesh's tetrahedron table (k_poly_tets): the
        // same numbers as the two passes below, looked up instead of summed
        const uint32_t k0 = C.tetOff[cell], k1 = C.tetOff[cell + 1];
        if (k0 == k1) { px = cx; py = cy; pz = cz; return; }
        const double r = rng.raw() * C.tetCum[k1 - 1];
        // the first tetrahedron whose running sum is not below r, else the last:
        // !(sum < r) holds from some index on, since the sums never decrease and
        // a NaN sum stays NaN
        uint32_t lo = k0, hi = k1 - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (C.tetCum[mid] < r) lo = mid + 1; else hi = mid;
        }
        const uint2 at = C.tetAT[lo];
        v0 = C.fvi[at.x]; v1 = C.fvi[at.y]; v2 = C.fvi[at.y + 1];
    } else {
        const uint32_t k0 = C.cfo[cell], k1 = C.cfo[cell + 1];
        double total = 0.0;
        uint32_t ntri = 0;
        for (uint32_t q = k0; q < k1; ++q) {
            const uint32_t f = C.cfFace[q], a = C.fvo[f], b = C.fvo[f + 1];
            if (b - a < 3) continue;
            for (uint32_t t = a + 1; t + 1 < b; ++t) {
                total += poly_tet_volume(C, C.fvi[a], C.fvi[t], C.fvi[t + 1], cx, cy, cz);
                ++ntri;
            }
        }
        if (ntri == 0) { px = cx; py = cy; pz = cz; return; }
        const double r = rng.raw() * total;
        // the first triangle whose running sum is not below r, else the last
        bool found = false;
        double run = 0.0;
        for (uint32_t q = k0; q < k1 && !found; ++q) {
            const uint32_t f = C.cfFace[q], a = C.fvo[f], b = C.fvo[f + 1];
            if (b - a < 3) continue;
            for (uint32_t t = a + 1; t + 1 < b; ++t) {
                run += poly_tet_volume(C, C.fvi[a], C.fvi[t], C.fvi[t + 1], cx, cy, cz);
                v0 = C.fvi[a]; v1 = C.fvi[t]; v2 = C.fvi[t + 1];
                if (!(run < r)) { found = true; break; }
            }
        }
    }
    double s = rng.raw(), t = rng.raw(), u = rng.raw(), tmp;
    if (s > t) { tmp = s; s = t; t = tmp; }
    if (t > u) { tmp = t; t = u; u = tmp; }
    if (s > t) { tmp = s; s = t; t = tmp; }
    const double a0 = s, a1 = t - s, a2 = u - t, a3 = 1 - u;
    px = a0 * C.vtx[3 * v0] + a1 * C.vtx[3 * v1] + a2 * C.vtx[3 * v2] + a3 * cx;
    py = a0 * C.vtx[3 * v0 + 1] + a1 * C.vtx[3 * v1 + 1] + a2 * C.vtx[3 * v2 + 1] + a3 * cy;
    pz = a0 * C.vtx[3 * v0 + 2] + a1 * C.vtx[3 * v1 + 2] + a2 * C.vtx[3 * v2 + 2] + a3 * cz;
}

// The table sample_in_poly_cell looks up: per cell its fan tetrahedra in the
// sampler's order, each with the running sum of the volumes up to it, formed by
// the sampler's own operations in its order (so equal to its sums bit for bit),
// and its (first, t) offsets into fvi.  tetOff comes from the host.
__global__ void k_poly_tets(Ctx C, const uint32_t *tetOff, double *tetCum, uint2 *tetAT) {
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < C.ncells; cell += gridDim.x * blockDim.x) {
        const double cx = C.mpx[cell], cy = C.mpy[cell], cz = C.mpz[cell];
        uint32_t o = tetOff[cell];
        double total = 0.0;
        for (uint32_t q = C.cfo[cell]; q < C.cfo[cell + 1]; ++q) {
            const uint32_t f = C.cfFace[q], a = C.fvo[f], b = C.fvo[f + 1];
            if (b - a < 3) continue;
            for (uint32_t t = a + 1; t + 1 < b; ++t) {
                total += poly_tet_volume(C, C.fvi[a], C.fvi[t], C.fvi[t + 1], cx, cy, cz);
                tetCum[o] = total;
                tetAT[o] = make_uint2(a, t);
                ++o;
            }
        }
    }
}

// the cell's mesh point (GetMeshPoint)
__device__ __forceinline__ void mesh_point(const Ctx &C, uint32_t c, double &mx, double &my, double &mz) {
    if (C.poly) { mx = C.mpx[c]; my = C.mpy[c]; mz = C.mpz[c]; return; }
    uint32_t i, j, k;
    cell_ijk(C, c, i, j, k);
    mx = C.xc[i]; my = C.yc[j]; mz = C.zc[k];
}

// RandomPointOnFace (utils/RandomOnFace.hpp:15-66) for a quad face.
template <class RNG>
__device__ inline void point_on_face(const double q[4][3], RNG &rng, double &px, double &py, double &pz) {
    double cum[2];
    double total = 0;
#pragma unroll
    for (int t = 1; t < 3; ++t) {
        double ux = q[t][0] - q[0][0], uy = q[t][1] - q[0][1], uz = q[t][2] - q[0][2];
        double vx = q[t + 1][0] - q[0][0], vy = q[t + 1][1] - q[0][1], vz = q[t + 1][2] - q[0][2];
        double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
        total += sqrt(cx * cx + cy * cy + cz * cz);
        cum[t - 1] = total;
    }
    double r = rng.raw() * total;
    int idx = (cum[0] < r) ? 1 : 0;   // lower_bound over two entries
    if (idx == 1 && cum[1] < r) idx = 2;
    if (idx >= 2) idx = 1;
    double r1 = rng.raw(), r2 = rng.raw();
    if (r1 + r2 > 1) { r1 = 1 - r1; r2 = 1 - r2; }
    const double a0 = 1 - r1 - r2;
    px = a0 * q[0][0] + r1 * q[idx + 1][0] + r2 * q[idx + 2][0];
    py = a0 * q[0][1] + r1 * q[idx + 1][1] + r2 * q[idx + 2][1];
    pz = a0 * q[0][2] + r1 * q[idx + 1][2] + r2 * q[idx + 2][2];
}

// RandomPointOnFace (utils/RandomOnFace.hpp:15-66) for polygon f of a
// polyhedral mesh: the fan triangles (v0, v_t, v_t+1) picked by area (the
// first whose cumulative area reaches u * total), then a folded barycentric
// point.  The cumulative areas are recomputed on the second pass with the same
// operations, so the pick sees the same numbers the total came from.
template <class RNG>
__device__ inline void point_on_polygon(const Ctx &C, uint32_t f, RNG &rng, double &px, double &py, double &pz) {
    const uint32_t a = C.fvo[f], nv = C.fvo[f + 1] - a;
    const double *v0 = C.vtx + 3 * static_cast<size_t>(C.fvi[a]);
    auto tri_area = [&](uint32_t t) {
        const double *v1 = C.vtx + 3 * static_cast<size_t>(C.fvi[a + t]);
        const double *v2 = C.vtx + 3 * static_cast<size_t>(C.fvi[a + t + 1]);
        const double ux = v1[0] - v0[0], uy = v1[1] - v0[1], uz = v1[2] - v0[2];
        const double vx = v2[0] - v0[0], vy = v2[1] - v0[1], vz = v2[2] - v0[2];
        const double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
        return sqrt(cx * cx + cy * cy + cz * cz);
    };
    double total = 0.0;
    for (uint32_t t = 1; t + 1 < nv; ++t) total += tri_area(t);
    const double r = rng.raw() * total;
    uint32_t idx = nv - 3;   // the last triangle when rounding leaves r above every cumulative area
    double cum = 0.0;
    for (uint32_t t = 1; t + 1 < nv; ++t) {
        cum += tri_area(t);
        if (!(cum < r)) { idx = t - 1; break; }
    }
    double r1 = rng.raw(), r2 = rng.raw();
    if (r1 + r2 > 1) { r1 = 1 - r1; r2 = 1 - r2; }
    const double a0 = 1 - r1 - r2;
    const double *v1 = C.vtx + 3 * static_cast<size_t>(C.fvi[a + idx + 1]);
    const double *v2 = C.vtx + 3 * static_cast<size_t>(C.fvi[a + idx + 2]);
    px = a0 * v0[0] + r1 * v1[0] + r2 * v2[0];
    py = a0 * v0[1] + r1 * v1[1] + r2 * v2[1];
    pz = a0 * v0[2] + r1 * v1[2] + r2 * v2[2];
}

__device__ __forceinline__ bool outside_box(const Ctx &C, double x, double y, double z) {
    return x < C.X0 || x > C.X1 || y < C.Y0 || y > C.Y1 || z < C.Z0 || z > C.Z1;
}

// outside-box repair of generateSingleParticle (radiation/RadiationIMC.hpp:2528-2541)
// and TwoSidesTemperature (boundary/TwoSidesTemperature.hpp:178-189)
__device__ __forceinline__ void repair_outside(const Ctx &C, double &x, double &y, double &z, double mx, double my,
                                               double mz) {
    if (!outside_box(C, x, y, z)) return;
    const double ox = x, oy = y, oz = z, dx = mx - ox, dy = my - oy, dz = mz - oz;
    double t = 1e-8;
    int guard = 0;
    while (outside_box(C, x, y, z) && t < 1.0 && guard++ < 64) {
        x = ox + t * dx; y = oy + t * dy; z = oz + t * dz;
        t *= 2;
    }
    x = x + 1e-8 * (mx - x);
    y = y + 1e-8 * (my - y);
    z = z + 1e-8 * (mz - z);
}

// ------------------------------------------------------------------ cell emission
// generateParticles per-photon loop (radiation/RadiationIMC.hpp:2405-2506) with
// generateSingleParticle (:2516-2553).  Packet e of cell c draws from stream
// (TAG_CELL_EMIT, step, e): 4 position, 2 direction, 1 time.  The launch makes
// packets e in [eBegin, eBegin + count) (a particle shard's range; the whole
// step's packets unsharded): packet e goes to bank slot bankBase + (e - eBegin)
// with pid pidBase + e.
// The cell of emitted packet e: the last cell whose offset is <= e (offsets
// has ncells + 1 entries, offsets[ncells] the total).  The lanes of a warp
// hold consecutive packets: the first active lane searches, the others walk
// forward from its cell over the few cells their packets are in (a lane that
// meets a long run of cells without packets searches the rest).
__device__ __forceinline__ uint32_t last_offset_at_most(const uint64_t *offsets, uint32_t lo, uint32_t hi, uint64_t e) {
    while (lo < hi) {   // the first index in [lo, hi) whose offset exceeds e
        const uint32_t mid = (lo + hi) >> 1;
        if (offsets[mid] <= e) lo = mid + 1; else hi = mid;
    }
    return lo - 1;
}
__device__ __forceinline__ uint32_t emission_cell(const uint64_t *offsets, uint32_t ncells, uint64_t e) {
    const unsigned m = __activemask();
    const int leader = __ffs(m) - 1;
    uint32_t c = 0;
    if (static_cast<int>(threadIdx.x & 31) == leader) c = last_offset_at_most(offsets, 0, ncells, e);
    c = __shfl_sync(m, c, leader);   // the leader's packet is the warp's first, so its cell is at or below ours
    for (int walk = 0; c + 1 < ncells && offsets[c + 1] <= e; ++walk) {
        if (walk == 32) return last_offset_at_most(offsets, c + 1, ncells, e);
        ++c;
    }
    return c;
}

__global__ void k_emit_cells(Ctx C, CellArrays A, const uint64_t *offsets, uint64_t eBegin, uint64_t count, Bank b,
                             uint32_t bankBase, uint32_t pidBase, double dt, DevStats *st) {
    double esum = 0.0;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = eBegin + j;
        const uint32_t c = emission_cell(offsets, C.ncells, e);
        const uint64_t np = A.photons[c];
        const double energyPerPhoton = A.emitE[c] * 1.0 / static_cast<double>(np);
        PhiloxRng rng;
        rng.init(C.seedLo, C.seedHi, TAG_CELL_EMIT, C.step, static_cast<uint32_t>(e), 0);
        PartReg p;
        p.cell = c;
        if (C.poly) sample_in_poly_cell(C, c, rng, p.x, p.y, p.z);
        else sample_in_cell(C, c, rng, p.x, p.y, p.z);
        double mx, my, mz;
        mesh_point(C, c, mx, my, mz);
        repair_outside(C, p.x, p.y, p.z, mx, my, mz);
        isotropic(rng, C.clight, p.vx, p.vy, p.vz);
        p.t = dt * rng.open();
        p.nu = 0.0;
        // moving material: the packet is emitted isotropically in the comoving
        // frame; its lab weight and frequency carry the Doppler factor (:2483-2493)
        const double D = C.withHydro ? doppler_shift(C, C.vel[c], p.vx, p.vy, p.vz) : 1.0;
        if (C.groups >= 2) {   // GetThermalEnergy (radiation/RadiationIMC.hpp:2495-2500)
            p.nu = mg_thermal_energy(C, c, rng.open());
            if (p.nu < 0.0) raise_error(C, STORM_DERR_MG_SAMPLE, c, static_cast<uint32_t>(e));
            if (C.withHydro) p.nu = p.nu / D;
        }
        p.w = C.withHydro ? A.emitE[c] / (static_cast<double>(np) * D) : energyPerPhoton;
        p.w0 = fabs(p.w);
        store_any(C, b, bankBase + static_cast<uint32_t>(j), p, pidBase + static_cast<uint32_t>(e), 0);
        esum += p.w;
    }
    esum = warp_sum(esum);
    if ((threadIdx.x & 31) == 0 && esum != 0.0) atomicAdd(&st->eEmitted, esum);
}

// The same packets in the FP32-tracking form: the cell's 12 fan tetrahedra
// have equal volume (a box), so the pick is floor(12 u); the point and the
// direction are drawn in the cell's own FP32 frame with the same draws in the
// same order (4 position, 2 direction, 1 time); time and weight stay FP64.
__device__ __forceinline__ void local_face_vertex(int side, int v, float hx, float hy, float hz, float &x, float &y,
                                                  float &z) {
    // vertex v of side `side` in face_vertices' order, relative to the cell centre
    const int axis = side >> 1;
    const float sgn = (side & 1) ? 1.0f : -1.0f;
    const float a = (v == 1 || v == 2) ? 1.0f : -1.0f;   // first in-plane coordinate
    const float b = (v >= 2) ? 1.0f : -1.0f;             // second in-plane coordinate
    if (axis == 0) { x = sgn * hx; y = a * hy; z = ((v == 2 || v == 3) ? 1.0f : -1.0f) * hz; }
    else if (axis == 1) { x = b * hx; y = sgn * hy; z = ((v == 1 || v == 2) ? 1.0f : -1.0f) * hz; }
    else { x = a * hx; y = ((v >= 2) ? 1.0f : -1.0f) * hy; z = sgn * hz; }
}

__global__ void k_emit_cells32(Ctx C, CellArrays A, const uint64_t *offsets, uint64_t eBegin, uint64_t count, Bank b,
                               uint32_t bankBase, uint32_t pidBase, double dt, DevStats *st) {
    double esum = 0.0;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = eBegin + j;
        const uint32_t c = emission_cell(offsets, C.ncells, e);
        const uint64_t np = A.photons[c];
        const double energyPerPhoton = A.emitE[c] * 1.0 / static_cast<double>(np);
        PhiloxRng rng;
        rng.init(C.seedLo, C.seedHi, TAG_CELL_EMIT, C.step, static_cast<uint32_t>(e), 0);
        Track32 T;
        T.cell = c;
        cell_ijk(C, c, T.i, T.j, T.k);
        const float hx = C.hx[T.i], hy = C.hy[T.j], hz = C.hz[T.k];
        const int tet = min(static_cast<int>(12.0f * rng.rawf()), 11);
        float s0 = rng.rawf(), s1 = rng.rawf(), s2 = rng.rawf(), tmp;
        if (s0 > s1) { tmp = s0; s0 = s1; s1 = tmp; }
        if (s1 > s2) { tmp = s1; s1 = s2; s2 = tmp; }
        if (s0 > s1) { tmp = s0; s0 = s1; s1 = tmp; }
        const int side = tet >> 1, tri = (tet & 1) + 1;
        float x0, y0, z0, x1, y1, z1, x2, y2, z2;
        local_face_vertex(side, 0, hx, hy, hz, x0, y0, z0);
        local_face_vertex(side, tri, hx, hy, hz, x1, y1, z1);
        local_face_vertex(side, tri + 1, hx, hy, hz, x2, y2, z2);
        const float a0 = s0, a1 = s1 - s0, a2 = s2 - s1;   // the centre's weight 1 - s2 multiplies 0
        T.qx = clampf(a0 * x0 + a1 * x1 + a2 * x2, hx);
        T.qy = clampf(a0 * y0 + a1 * y1 + a2 * y2, hy);
        T.qz = clampf(a0 * z0 + a1 * z1 + a2 * z2, hz);
        const float theta = 6.2831853f * rng.rawf();
        const float cz = 2.0f * rng.rawf() - 1.0f;
        const float sz = sqrtf(fmaxf(0.0f, 1.0f - cz * cz));
        float sth, cth;
        __sincosf(theta, &sth, &cth);
        T.ux = sz * cth; T.uy = sz * sth; T.uz = cz;
        T.t = dt * rng.open();
        T.w = energyPerPhoton;
        T.w0 = fabs(T.w);
        const uint32_t slot = bankBase + static_cast<uint32_t>(j);
        store32(b, slot, T, pidBase + static_cast<uint32_t>(e), 0);
        if (C.groups >= 2) {   // GetThermalEnergy (radiation/RadiationIMC.hpp:2495-2500)
            const double nu = mg_thermal_energy(C, c, rng.open());
            if (nu < 0.0) raise_error(C, STORM_DERR_MG_SAMPLE, c, static_cast<uint32_t>(e));
            store_nu32(b, slot, static_cast<float>(nu));
        }
        esum += T.w;
    }
    esum = warp_sum(esum);
    if ((threadIdx.x & 31) == 0 && esum != 0.0) atomicAdd(&st->eEmitted, esum);
}

// ------------------------------------------------------------------ face emission
// SideTemperature / TwoSidesTemperature::generateNewBoundaryParticles
// (boundary/SideTemperature.hpp:114-163, TwoSidesTemperature.hpp:126-199) for the
// per-face descriptor.  Face packet f draws from (TAG_FACE_EMIT, step, f):
// 3 position, mu, theta, time.
__global__ void k_emit_faces(Ctx C, FaceSources F, uint64_t fBegin, uint64_t count, Bank b, uint32_t bankBase,
                             uint32_t pidBase, double dt, DevStats *st) {
    double esum = 0.0;
    for (uint64_t slot = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; slot < count;
         slot += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t f = fBegin + slot;
        uint32_t lo = 0, hi = F.count;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (F.offset[mid] <= f) lo = mid + 1; else hi = mid;
        }
        const uint32_t q = lo - 1;
        const uint32_t c = F.cell[q];
        const int side = F.side[q];
        const int axis = side >> 1;
        const double sgn = (side & 1) ? -1.0 : 1.0;
        const uint64_t Np = F.offset[q + 1] - F.offset[q];
        const double Tf = C.sourceT[side];
        const double T4 = (Tf * Tf) * (Tf * Tf);
        uint32_t i, j, k;
        cell_ijk(C, c, i, j, k);
        double area;   // Grid::GetArea
        if (C.poly) {
            area = F.area[q];
        } else {
            const double dx = C.xe[i + 1] - C.xe[i], dy = C.ye[j + 1] - C.ye[j], dz = C.ze[k + 1] - C.ze[k];
            area = axis == 0 ? dy * dz : (axis == 1 ? dz * dx : dx * dy);
        }
        const double energy = C.sigmaSB * T4 * area * dt / static_cast<double>(Np);
        PhiloxRng rng;
        rng.init(C.seedLo, C.seedHi, TAG_FACE_EMIT, C.step, static_cast<uint32_t>(f), 0);
        PartReg p;
        if (C.poly) {
            point_on_polygon(C, F.face[q], rng, p.x, p.y, p.z);
        } else {
            double qv[4][3];
            face_vertices(C, i, j, k, side, qv);
            point_on_face(qv, rng, p.x, p.y, p.z);
        }
        const double mu = sqrt(rng.raw());
        double v[3];
        v[axis] = sgn * mu;
        const double one_m = sqrt(1 - mu * mu);
        const double theta = 2 * 3.14159265358979323846 * rng.raw();
        double stt, ctt;
        sincos(theta, &stt, &ctt);
        v[(axis + 1) % 3] = one_m * ctt;
        v[(axis + 2) % 3] = one_m * stt;
        p.vx = v[0] * C.clight; p.vy = v[1] * C.clight; p.vz = v[2] * C.clight;
        p.w = energy;
        p.nu = 0.0;   // gray problems carry frequency 0
        p.t = dt * rng.raw();
        if (C.groups >= 2) {
            // DensmoreBoundary::generateNewBoundaryParticles
            // (examples/densmore2012/DensmoreBoundary.hpp:128-139): the first group
            // whose cumulative Planck integral reaches u * total (the last group
            // when none does), then a uniform energy inside it; two draws after
            // the time draw, so gray streams are unchanged.
            const uint32_t G = C.groups;
            const double *row = C.faceCdf + static_cast<size_t>(side) * (G + 1);
            const double total = row[G];
            if (total > 0.0) {
                const double r = rng.raw() * total;
                uint32_t lo = 0, hi = G - 1;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (row[mid + 1] < r) lo = mid + 1; else hi = mid;
                }
                p.nu = C.gb[lo] + rng.raw() * (C.gb[lo + 1] - C.gb[lo]);
            } else {
                p.nu = 0.5 * (C.gb[0] + C.gb[G]);
            }
        }
        p.cell = c;
        double mx, my, mz;
        mesh_point(C, c, mx, my, mz);
        repair_outside(C, p.x, p.y, p.z, mx, my, mz);
        p.w0 = fabs(p.w);
        store_any(C, b, bankBase + static_cast<uint32_t>(slot), p, pidBase + static_cast<uint32_t>(f), 0);
        esum += p.w;
    }
    esum = warp_sum(esum);
    if ((threadIdx.x & 31) == 0 && esum != 0.0) atomicAdd(&st->eEmitted, esum);
}

// The Planck spectrum of each box face over the groups, cumulative
// planck_integral(b_g / kT, b_{g+1} / kT) at kT = k_B T_face, as
// DensmoreBoundary builds it (examples/densmore2012/DensmoreBoundary.hpp:99-109).
// One thread per face; rebuilt only when a face temperature changes.
__global__ void k_face_spectra(Ctx C, double *cdf) {
    const int f = threadIdx.x;
    if (f >= 6) return;
    const uint32_t G = C.groups;
    double *row = cdf + static_cast<size_t>(f) * (G + 1);
    const double kT = C.kBoltz * C.sourceT[f];
    double acc = 0.0;
    row[0] = 0.0;
    for (uint32_t g = 0; g < G; ++g) {
        if (kT > 0.0) {
            const double a = C.gb[g] / kT, b = C.gb[g + 1] / kT;
            acc += (a > 0.0 && b > a) ? planck_integral(a, b) : 0.0;
        }
        row[g + 1] = acc;
    }
}

// ------------------------------------------------------------------ transport
struct BlockStats {
    unsigned long long segments, rwSteps, escaped, cutoff, census;
    double eDeposited, eEscaped, eCensusPre;
};

__device__ __forceinline__ void block_stats_zero(BlockStats &bs) {
    if (threadIdx.x == 0) bs = BlockStats{0, 0, 0, 0, 0, 0.0, 0.0, 0.0};
    __syncthreads();
}

// One warp's share of the step statistics: reduced over the warp with shuffles,
// then one shared atomic per quantity.  Every lane of the warp calls it.
__device__ __forceinline__ void warp_stats(BlockStats &bs, uint32_t segs, uint32_t rw, double dep, int outcome,
                                           double w) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t s = warp_sum(segs);
    const unsigned mE = __ballot_sync(FULL, outcome == OUT_ESCAPE);
    const unsigned mX = __ballot_sync(FULL, outcome == OUT_CUTOFF);
    const unsigned mC = __ballot_sync(FULL, outcome == OUT_CENSUS);
    const uint32_t r = __any_sync(FULL, rw != 0) ? warp_sum(rw) : 0u;
    const double d = __any_sync(FULL, dep != 0.0) ? warp_sum(dep) : 0.0;
    const double eE = mE ? warp_sum(outcome == OUT_ESCAPE ? w : 0.0) : 0.0;
    const double eC = mC ? warp_sum(outcome == OUT_CENSUS ? w : 0.0) : 0.0;
    if (lane == 0) {
        if (s) atomicAdd(&bs.segments, static_cast<unsigned long long>(s));
        if (r) atomicAdd(&bs.rwSteps, static_cast<unsigned long long>(r));
        if (d != 0.0) atomicAdd(&bs.eDeposited, d);
        if (mE) { atomicAdd(&bs.escaped, static_cast<unsigned long long>(__popc(mE))); atomicAdd(&bs.eEscaped, eE); }
        if (mX) atomicAdd(&bs.cutoff, static_cast<unsigned long long>(__popc(mX)));
        if (mC) { atomicAdd(&bs.census, static_cast<unsigned long long>(__popc(mC))); atomicAdd(&bs.eCensusPre, eC); }
    }
}

__device__ __forceinline__ void block_stats_flush(const BlockStats &bs, DevStats *st) {
    __syncthreads();
    if (threadIdx.x == 0) {
        if (bs.segments) atomicAdd(&st->segments, bs.segments);
        if (bs.rwSteps) atomicAdd(&st->rwSteps, bs.rwSteps);
        if (bs.escaped) atomicAdd(&st->escaped, bs.escaped);
        if (bs.cutoff) atomicAdd(&st->cutoff, bs.cutoff);
        if (bs.census) atomicAdd(&st->census, bs.census);
        if (bs.eDeposited != 0.0) atomicAdd(&st->eDeposited, bs.eDeposited);
        if (bs.eEscaped != 0.0) atomicAdd(&st->eEscaped, bs.eEscaped);
        if (bs.eCensusPre != 0.0) atomicAdd(&st->eCensusPre, bs.eCensusPre);
    }
}

// The two particle forms behind one interface: the FP64 form (global FP64
// coordinates, the reference's arithmetic) and the FP32-tracking form.
// Form64T<0> is the gray FP64 form without DDMC on a Cartesian grid;
// Form64T<1> adds the multigroup and DDMC branches; Form64T<2> runs on a
// convex-polyhedral mesh and Form64T<5> is it with the DDMC branch;
// Form64T<4> is Form64T<1> without the DDMC branch.  Problems without
// withDDMC run the variants without it: less code for the instruction cache,
// whose misses bound the multigroup and polyhedral kernels.  TL is the
// tally: SegmentTallyEg adds the group time averages (withEgTimeAvg),
// SegmentTallyFixed sums in fixed point (reproducible tallies).
template <int V, class TL = SegmentTally>
struct Form64T {
    using T = Track;
    using Rng = PhiloxRng;
    using Tally = TL;
    static __device__ __forceinline__ void load(const Ctx &C, const Bank &b, uint32_t q, T &t) {
        load_part(b, q, t.p);
        track_begin(C, t);
    }
    static __device__ __forceinline__ void keep(const Bank &b, uint32_t q, const T &t, uint32_t pid, uint32_t draw) {
        store_part(b, q, t.p, pid, draw);
    }
    static __device__ __forceinline__ void store(const CensusBank &b, uint32_t q, const T &t, uint32_t pid,
                                                 uint32_t draw) {
        census_store64(b, q, t.p, pid, draw);
    }
    template <class RNG, class TALLY>
    static __device__ __forceinline__ int seg(const Ctx &C, T &t, RNG &rng, TALLY &tal, int &usedRW, int &err) {
        PhysOut o = physics_step<V>(C, t, rng, tal);
        if (o.errCode) { err = o.errCode; return OUT_ERROR; }
        usedRW = o.usedRW == 1;   // Random Walk jumps (2 marks a DDMC step)
        int m = manager_handle<V == 2 || V == 5>(C, t, o);
        if (m == OUT_ERROR) err = STORM_DERR_NOT_ON_BOUNDARY;
        return m;
    }
    static __device__ __forceinline__ uint32_t cell(const T &t) { return t.p.cell; }
    static __device__ __forceinline__ double weight(const T &t) { return t.p.w; }
};
using Form64 = Form64T<0>;
using Form64Full = Form64T<1>;
using Form64Poly = Form64T<2>;
using Form64PolyDDMC = Form64T<5>;   // Form64Poly with the DDMC branch
using Form64Hydro = Form64T<3>;   // Form64Full with moving material
using Form64MG = Form64T<4>;      // Form64Full without the DDMC branch
using Form64FullEg = Form64T<1, SegmentTallyEg>;   // the multigroup forms with the group time averages
using Form64MGEg = Form64T<4, SegmentTallyEg>;
using Form64HydroEg = Form64T<3, SegmentTallyEg>;
using Form64Fix = Form64T<0, SegmentTallyFixed>;   // reproducible tallies
using Form64FullFix = Form64T<1, SegmentTallyFixed>;
using Form64MGFix = Form64T<4, SegmentTallyFixed>;
using Form64PolyFix = Form64T<2, SegmentTallyFixed>;
using Form64PolyDDMCFix = Form64T<5, SegmentTallyFixed>;
template <bool POLY, bool DDMC = true, class TL = SegmentTally>
struct Form32T {
    using T = Track32;
    using Rng = PhiloxRng4;
    using Tally = TL;
    static __device__ __forceinline__ void load(const Ctx &C, const Bank &b, uint32_t q, T &t) {
        load32(b, q, t);
        cell_ijk(C, t.cell, t.i, t.j, t.k);
        t.cc = OUTSIDE;
    }
    static __device__ __forceinline__ void keep(const Bank &b, uint32_t q, const T &t, uint32_t pid, uint32_t draw) {
        store32(b, q, t, pid, draw);
    }
    static __device__ __forceinline__ void store(const CensusBank &b, uint32_t q, const T &t, uint32_t pid,
                                                 uint32_t draw) {
        census_store32(b, q, t, pid, draw);
    }
    template <class RNG, class TALLY>
    static __device__ __forceinline__ int seg(const Ctx &C, T &t, RNG &rng, TALLY &tal, int &usedRW, int &err) {
        int m = segment32<false, RNG, TALLY, POLY, DDMC>(C, t, rng, tal, usedRW, err);
        if (m == OUT_ERROR && !err) err = STORM_DERR_NOT_ON_BOUNDARY;
        return m;
    }
    static __device__ __forceinline__ uint32_t cell(const T &t) { return t.cell; }
    static __device__ __forceinline__ double weight(const T &t) { return t.w; }
};
using Form32 = Form32T<false>;
using Form32Lean = Form32T<false, false>;   // without the DDMC branch
using Form32Poly = Form32T<true, false>;   // without the DDMC branch
using Form32PolyDDMC = Form32T<true, true>;
using Form32Fix = Form32T<false, true, SegmentTallyFixed>;   // reproducible tallies
using Form32LeanFix = Form32T<false, false, SegmentTallyFixed>;
using Form32PolyFix = Form32T<true, false, SegmentTallyFixed>;
using Form32PolyDDMCFix = Form32T<true, true, SegmentTallyFixed>;
// The FP32-tracking form of a multigroup problem: the frequency rides along.
template <bool DDMC = true, class TL = SegmentTally>
struct Form32MGT {
    using T = Track32;
    using Rng = PhiloxRng4;
    using Tally = TL;
    static __device__ __forceinline__ void load(const Ctx &C, const Bank &b, uint32_t q, T &t) {
        load32(b, q, t);
        t.nu = load_nu32(b, q);
        cell_ijk(C, t.cell, t.i, t.j, t.k);
        t.cc = OUTSIDE;
    }
    static __device__ __forceinline__ void keep(const Bank &b, uint32_t q, const T &t, uint32_t pid, uint32_t draw) {
        store32(b, q, t, pid, draw);
        store_nu32(b, q, t.nu);
    }
    static __device__ __forceinline__ void store(const CensusBank &b, uint32_t q, const T &t, uint32_t pid,
                                                 uint32_t draw) {
        census_store32_mg(b, q, t, pid, draw);
    }
    template <class RNG, class TALLY>
    static __device__ __forceinline__ int seg(const Ctx &C, T &t, RNG &rng, TALLY &tal, int &usedRW, int &err) {
        int m = segment32<true, RNG, TALLY, false, DDMC>(C, t, rng, tal, usedRW, err);
        if (m == OUT_ERROR && !err) err = STORM_DERR_NOT_ON_BOUNDARY;
        return m;
    }
    static __device__ __forceinline__ uint32_t cell(const T &t) { return t.cell; }
    static __device__ __forceinline__ double weight(const T &t) { return t.w; }
};
using Form32MG = Form32MGT<true>;
using Form32MGLean = Form32MGT<false>;   // without the DDMC branch
using Form32MGEg = Form32MGT<true, SegmentTallyEg>;   // with the group time averages
using Form32MGLeanEg = Form32MGT<false, SegmentTallyEg>;
using Form32MGFix = Form32MGT<true, SegmentTallyFixed>;   // reproducible tallies
using Form32MGLeanFix = Form32MGT<false, SegmentTallyFixed>;

// One bank visit of the HandleAll loop (manager/MonteCarloManagerSerial.hpp:267-383):
// every active particle runs up to K segments in registers; survivors are
// compacted into the next bank and census particles appended to the census bank
// (warp ballot + one atomic per warp).  Step statistics are reduced per warp.
template <class F>
__device__ __forceinline__ void visit_bank(const Ctx &C, const Bank &in, uint32_t n, const Bank &out, uint32_t *nOut,
                                           const CensusBank &cen, uint32_t *nCen, uint32_t K, BlockStats &bs) {
    const unsigned lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t idx = base + threadIdx.x;
        const bool active = idx < n;
        typename F::T t;
        uint32_t pid = 0, draw = 0, s = 0, rw = 0;
        double dep = 0.0, w = 0.0;
        int outcome = OUT_CONTINUE;
        if (active) {
            F::load(C, in, idx, t);
            pid = in.pid[idx];
            typename F::Rng rng;
            rng.init(C.seedLo, C.seedHi, TAG_TRANSPORT, C.step, pid, in.draw[idx]);
            SegmentTally tal;
            tal.init(C.eint, C.eradAvg, C.perCellCounters ? C.segs : nullptr);
            while (s < K) {
                const uint32_t cell0 = F::cell(t);
                tal.enter(cell0);
                ++s;
                int usedRW = 0, err = 0;
                outcome = F::seg(C, t, rng, tal, usedRW, err);
                rw += usedRW;
                if (outcome != OUT_CONTINUE) {
                    if (outcome == OUT_ERROR) raise_error(C, err, cell0, pid);
                    break;
                }
            }
            dep = tal.depSum;
            draw = rng.draw;
            w = F::weight(t);
        }
        warp_stats(bs, s, rw, dep, outcome, w);
        const bool keep = active && outcome == OUT_CONTINUE;
        const bool cens = active && outcome == OUT_CENSUS;
        const unsigned mK = __ballot_sync(FULL, keep), mC = __ballot_sync(FULL, cens);
        uint32_t bK = 0, bC = 0;
        if (lane == 0) {
            if (mK) bK = atomicAdd(nOut, __popc(mK));
            if (mC) bC = atomicAdd(nCen, __popc(mC));
        }
        bK = __shfl_sync(FULL, bK, 0);
        bC = __shfl_sync(FULL, bC, 0);
        const unsigned lt = lanemask_lt();
        if (keep) F::keep(out, bK + __popc(mK & lt), t, pid, draw);
        if (cens) F::store(cen, bC + __popc(mC & lt), t, pid, draw);
    }
}

template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_transport(Ctx C, Bank in, const uint32_t *nIn, Bank out,
                                                          uint32_t *nOut, CensusBank cen, uint32_t *nCen, uint32_t K,
                                                          DevStats *st) {
    __shared__ BlockStats bs;
    block_stats_zero(bs);
    visit_bank<Form64Full>(C, in, *nIn, out, nOut, cen, nCen, K, bs);
    block_stats_flush(bs, st);
}

// The same bank visit in the FP32-tracking form.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_transport32(Ctx C, Bank in, const uint32_t *nIn, Bank out,
                                                            uint32_t *nOut, CensusBank cen, uint32_t *nCen, uint32_t K,
                                                            DevStats *st) {
    __shared__ BlockStats bs;
    block_stats_zero(bs);
    visit_bank<Form32>(C, in, *nIn, out, nOut, cen, nCen, K, bs);
    block_stats_flush(bs, st);
}

// ------------------------------------------------------------------ persistent transport
// The whole HandleAll loop in one launch.  Every lane holds one history; a lane
// whose particle reaches census, escapes or is cut off writes it out and takes
// the next unstarted particle, so lanes do not idle behind the longest history
// of their warp.  Each warp takes unstarted particles from the bank in chunks of
// REFILL_CHUNK (one global atomic per chunk) and hands them to its empty lanes
// between bursts of `burst` segments.  Per-lane totals (segments, deposits,
// census energy) live in the lane's own shared-memory slot until the end.  A
// history longer than maxSegs raises STORM_DERR_HISTORY_CAP and stops.
constexpr uint32_t REFILL_CHUNK = 32;

template <class F, int MINB>
__global__ void __launch_bounds__(256, MINB) k_transport_refill(Ctx C, Bank in, uint32_t n, uint32_t *nextIdx, CensusBank cen,
                                                                 uint32_t *nCen, uint32_t burst, uint32_t maxSegs,
                                                                 DevStats *st) {
    __shared__ BlockStats bs;
    __shared__ double sDep[256], sCen[256];
    __shared__ uint32_t sSegs[256], sRw[256];
    const unsigned tid = threadIdx.x;
    sDep[tid] = 0.0; sCen[tid] = 0.0; sSegs[tid] = 0; sRw[tid] = 0;
    block_stats_zero(bs);
    const unsigned lane = tid & 31;
    const unsigned lt = lanemask_lt();
    typename F::T t;
    typename F::Rng rng;
    uint32_t pid = 0, segsThis = 0;
    bool has = false;
    uint32_t cBase = 0, cLeft = 0;   // warp-uniform: this warp's chunk of unstarted particles
    bool drained = false;            // warp-uniform: the bank counter has passed n
    for (;;) {
        unsigned need = __ballot_sync(FULL, !has);
        while (need) {
            if (cLeft == 0) {
                if (drained) break;
                uint32_t b = 0;
                if (lane == 0) b = atomicAdd(nextIdx, REFILL_CHUNK);
                b = __shfl_sync(FULL, b, 0);
                if (b >= n) { drained = true; break; }
                if (n - b <= REFILL_CHUNK) drained = true;
                cBase = b;
                cLeft = min(REFILL_CHUNK, n - b);
            }
            const uint32_t take = min(static_cast<uint32_t>(__popc(need)), cLeft);
            const uint32_t rank = __popc(need & lt);
            if (!has && rank < take) {
                const uint32_t q = cBase + rank;
                F::load(C, in, q, t);
                pid = in.pid[q];
                rng.init(C.seedLo, C.seedHi, TAG_TRANSPORT, C.step, pid, in.draw[q]);
                segsThis = 0;
                has = true;
            }
            cBase += take;
            cLeft -= take;
            need = __ballot_sync(FULL, !has);
        }
        if (!__any_sync(FULL, has)) break;
        int outcome = OUT_CONTINUE;
        if (has) {
            typename F::Tally tal;
            tal.init(C.eint, C.eradAvg, C.perCellCounters ? C.segs : nullptr);
            if constexpr (std::is_same_v<typename F::Tally, SegmentTallyFixed>) tal.init_fixed(C);
            uint32_t segs = 0, rws = 0;
            for (uint32_t b = 0; b < burst; ++b) {
                const uint32_t cell0 = F::cell(t);
                tal.enter(cell0);
                ++segs;
                int usedRW = 0, err = 0;
                outcome = F::seg(C, t, rng, tal, usedRW, err);
                rws += usedRW;
                if (outcome != OUT_CONTINUE) {
                    if (outcome == OUT_ERROR) raise_error(C, err, cell0, pid);
                    break;
                }
                if (++segsThis >= maxSegs) {
                    raise_error(C, STORM_DERR_HISTORY_CAP, cell0, pid);
                    outcome = OUT_ERROR;
                    break;
                }
            }
            sSegs[tid] += segs;
            if (rws) sRw[tid] += rws;
            sDep[tid] += tal.depSum;
            if (outcome == OUT_ESCAPE) { atomicAdd(&bs.escaped, 1ull); atomicAdd(&bs.eEscaped, F::weight(t)); }
            else if (outcome == OUT_CUTOFF) atomicAdd(&bs.cutoff, 1ull);
            else if (outcome == OUT_CENSUS) sCen[tid] += F::weight(t);
        }
        const bool cens = has && outcome == OUT_CENSUS;
        const unsigned mC = __ballot_sync(FULL, cens);
        if (mC) {
            uint32_t bC = 0;
            if (lane == 0) {
                bC = atomicAdd(nCen, __popc(mC));
                atomicAdd(&bs.census, static_cast<unsigned long long>(__popc(mC)));
            }
            bC = __shfl_sync(FULL, bC, 0);
            if (cens) F::store(cen, bC + __popc(mC & lt), t, pid, rng.draw);
        }
        if (has && outcome != OUT_CONTINUE) has = false;
    }
    // per-lane totals -> block
    const uint32_t segs = warp_sum(sSegs[tid]), rws = warp_sum(sRw[tid]);
    const double dep = warp_sum(sDep[tid]), eC = warp_sum(sCen[tid]);
    if (lane == 0) {
        if (segs) atomicAdd(&bs.segments, static_cast<unsigned long long>(segs));
        if (rws) atomicAdd(&bs.rwSteps, static_cast<unsigned long long>(rws));
        if (dep != 0.0) atomicAdd(&bs.eDeposited, dep);
        if (eC != 0.0) atomicAdd(&bs.eCensusPre, eC);
    }
    block_stats_flush(bs, st);
}

// ------------------------------------------------------------------ comb
// CombPopulationControl::activate (population/CombPopulationControl.hpp:79-253).
// Sort key = (cell << b) | keyed bijective hash of the particle's pid on b bits
// (every pid of the step is below 2^b): a pseudo-random
// order inside each cell (the reference sorts by id then std::shuffles) that does
// not depend on the order particles reached census.  Zero-weight particles get
// cell = Ncells and sort last (they are skipped, :136-137).
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
    return h;
}
// A keyed bijection of [0, 2^b): xor with the key, then odd multiplications and
// xor-shifts, each invertible modulo 2^b.  pid < 2^b, so (cell << b) | hash is a
// total order with no ties in b + cell bits.
__device__ __forceinline__ uint32_t comb_hash(uint32_t pid, uint32_t key, int b) {
    const uint32_t mask = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
    uint32_t h = (pid ^ key) & mask;
    h = (h * 0x9E3779B1u) & mask;
    h ^= h >> ((b + 1) / 2);
    h = (h * 0x85EBCA77u) & mask;
    h ^= h >> ((b + 2) / 3);
    h = (h * 0xC2B2AE3Du) & mask;
    h ^= h >> ((b + 1) / 2);
    return h;
}
// ------------------------------------------------------------------ particle shards
// The shard a pid belongs to: census pids by the shards' census ranges, then
// the step's cell packets and face packets, each cut into equal ranges.
// C.shardBounds holds the three sets of S + 1 pid bounds, one after the other.
__device__ __forceinline__ uint32_t shard_of_pid(const Ctx &C, uint32_t pid) {
    const uint32_t S = C.shards;
    const uint64_t *B = C.shardBounds;
    const uint64_t p = pid;
    const uint32_t g = p < B[S] ? 0u : (p < B[(S + 1) + S] ? 1u : 2u);
    const uint64_t *b = B + static_cast<size_t>(g) * (S + 1);
    uint32_t lo = 0, hi = S;   // the last shard whose first pid is <= p
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (b[mid] <= p) lo = mid; else hi = mid;
    }
    return lo;
}

// The cell of a comb run: runs are (shard, cell) when sharded, else (cell, bin).
__device__ __forceinline__ uint32_t cell_of_run(const Ctx &C, uint64_t run, uint32_t bins) {
    return C.shards > 1 ? static_cast<uint32_t>(run % C.ncells) : static_cast<uint32_t>(run / bins);
}

__global__ void k_comb_keys(Ctx C, CensusBank cen, uint32_t n, uint64_t *keys, uint32_t *vals, uint32_t combKey,
                            int pidBits, double *wc) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const double w = census_w(C, cen, q);
        if (wc) wc[q] = w;
        const uint2 cp = census_cell_pid(C, cen, q);
        const uint32_t pid = cp.y;
        uint32_t cell = cp.x;
        // FP32-tracking particles are inside their cell by construction
        if (!C.fp32) {
            const uint4 a = cen.rec[static_cast<size_t>(q) * 6], b = cen.rec[static_cast<size_t>(q) * 6 + 1];
            if (outside_box(C, lo_double(a), hi_double(a), lo_double(b))) raise_error(C, STORM_DERR_COMB_OUTSIDE, cell, pid);
        }
        const bool badWeight = !isfinite(w) || w < 0.0;
        if (badWeight) raise_error(C, STORM_DERR_COMB_WEIGHT, cell, pid);
        // zero, negative and non-finite weights never reach the per-cell loops
        if (w == 0.0 || badWeight || cell >= C.ncells) cell = C.ncells;
        // sharded: runs (shard, cell), shard-major; the excluded particles after every run
        uint64_t run = cell;
        if (C.shards > 1)
            run = cell >= C.ncells ? static_cast<uint64_t>(C.ncells) * C.shards
                                   : static_cast<uint64_t>(shard_of_pid(C, pid)) * C.ncells + cell;
        keys[q] = (run << pidBits) | comb_hash(pid, combKey, pidBits);
        vals[q] = q;
    }
}

// LSD radix sort, 8-bit digits: per-tile histograms, scan, stable scatter.
constexpr int RS_THREADS = 256, RS_WARPS = 8, RS_PER_WARP = 512, RS_TILE = RS_WARPS * RS_PER_WARP;

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const uint64_t *keys, uint32_t n, int shift, uint32_t *tileHist,
                                                        uint32_t ntiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * RS_TILE;
    for (int it = 0; it < RS_TILE / RS_THREADS; ++it) {
        uint32_t q = base + it * RS_THREADS + threadIdx.x;
        if (q < n) atomicAdd(&h[(keys[q] >> shift) & 255u], 1u);
    }
    __syncthreads();
    tileHist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// exclusive scan (in place) of the digit-major tile histogram, three phases
__global__ void k_scan32_tiles(uint32_t *v, uint32_t n, uint64_t *tileSums) {
    __shared__ uint64_t sh[32];
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t x = q < n ? v[q] : 0;
    uint64_t inc = block_scan_incl(x, sh);
    if (q < n) v[q] = static_cast<uint32_t>(inc - x);
    if (threadIdx.x == blockDim.x - 1) tileSums[blockIdx.x] = inc;
}
__global__ void k_scan32_add(uint32_t *v, uint32_t n, const uint64_t *tileSums) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) v[q] += static_cast<uint32_t>(tileSums[blockIdx.x]);
}

// exclusive scan of the digit-major tile histogram (256 * ntiles) by one block
__global__ void k_rs_scan(uint32_t *tileHist, uint32_t len) {
    __shared__ uint64_t sh[32];
    __shared__ uint64_t last;
    uint64_t carry = 0;
    for (uint32_t base = 0; base < len; base += blockDim.x) {
        uint32_t q = base + threadIdx.x;
        uint64_t v = q < len ? tileHist[q] : 0;
        uint64_t inc = block_scan_incl(v, sh);
        if (q < len) tileHist[q] = static_cast<uint32_t>(carry + inc - v);
        if (threadIdx.x == blockDim.x - 1) last = inc;
        __syncthreads();
        carry += last;
        __syncthreads();
    }
}

// Stable scatter of one 8-bit digit.  The block ranks its tile in shared memory
// (per-warp match_any counts, then a scan over digits), stages the tile there in
// digit order and writes it out in runs of equal digits, so global writes are
// coalesced within each run.
constexpr int RS_PER_THREAD = RS_PER_WARP / 32;
constexpr size_t RS_SMEM = static_cast<size_t>(RS_TILE) * 12 + RS_WARPS * 256 * 4 + 2 * 256 * 4;

__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const uint64_t *kin, const uint32_t *vin, uint64_t *kout,
                                                           uint32_t *vout, uint32_t n, int shift,
                                                           const uint32_t *tileOff, uint32_t ntiles) {
    extern __shared__ __align__(16) unsigned char rsMem[];
    __shared__ uint64_t scanSh[32];
    uint64_t *sk = reinterpret_cast<uint64_t *>(rsMem);
    uint32_t *sv = reinterpret_cast<uint32_t *>(rsMem + static_cast<size_t>(RS_TILE) * 8);
    uint32_t(*wc)[256] = reinterpret_cast<uint32_t(*)[256]>(rsMem + static_cast<size_t>(RS_TILE) * 12);
    uint32_t *dstart = reinterpret_cast<uint32_t *>(rsMem + static_cast<size_t>(RS_TILE) * 12 + RS_WARPS * 256 * 4);
    uint32_t *gbase = dstart + 256;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int d = lane; d < 256; d += 32) wc[wid][d] = 0;
    __syncwarp();
    const uint32_t tileBase = blockIdx.x * RS_TILE;
    const uint32_t start = tileBase + wid * RS_PER_WARP;
    const unsigned lt = lanemask_lt();
    uint64_t key[RS_PER_THREAD];
    uint32_t val[RS_PER_THREAD], rank[RS_PER_THREAD];
#pragma unroll
    for (int it = 0; it < RS_PER_THREAD; ++it) {
        const uint32_t q = start + it * 32 + lane;
        key[it] = q < n ? kin[q] : 0;
        val[it] = q < n ? vin[q] : 0;
    }
#pragma unroll
    for (int it = 0; it < RS_PER_THREAD; ++it) {
        const uint32_t q = start + it * 32 + lane;
        const uint32_t d = q < n ? static_cast<uint32_t>((key[it] >> shift) & 255u) : 256u;
        const unsigned m = __match_any_sync(FULL, d);
        const uint32_t before = d < 256u ? wc[wid][d] : 0u;
        __syncwarp();
        rank[it] = before + __popc(m & lt);
        if (d < 256u && (__ffs(m) - 1) == lane) wc[wid][d] = before + __popc(m);
        __syncwarp();
    }
    __syncthreads();
    {
        // digit d: per-warp exclusive offsets within the digit, then the digit's start in the tile
        const uint32_t d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) {
            const uint32_t c = wc[w][d];
            wc[w][d] = run;
            run += c;
        }
        const uint64_t incl = block_scan_incl(run, scanSh);
        dstart[d] = static_cast<uint32_t>(incl - run);
        gbase[d] = tileOff[d * ntiles + blockIdx.x];
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < RS_PER_THREAD; ++it) {
        const uint32_t q = start + it * 32 + lane;
        if (q < n) {
            const uint32_t d = static_cast<uint32_t>((key[it] >> shift) & 255u);
            const uint32_t pos = dstart[d] + wc[wid][d] + rank[it];
            sk[pos] = key[it];
            sv[pos] = val[it];
        }
    }
    __syncthreads();
    const uint32_t cnt = min(static_cast<uint32_t>(RS_TILE), n - tileBase);
    for (uint32_t pos = threadIdx.x; pos < cnt; pos += RS_THREADS) {
        const uint64_t k = sk[pos];
        const uint32_t d = static_cast<uint32_t>((k >> shift) & 255u);
        const uint32_t g = gbase[d] + (pos - dstart[d]);
        kout[g] = k;
        vout[g] = sv[pos];
    }
}

// ------------------------------------------------------------------ bucket sort of the comb keys
// The comb's keys are (run << pidBits) | hash, the hash a keyed bijection of
// the pid, so the keys of one run are distinct and their sorted order is
// unique.  Instead of an LSD radix sort over all run and pid bits, the keys are
// counted per run, placed in their run's range in arrival order (atomics), and
// each run is then sorted on its own in shared memory (bitonic).  The result
// is the radix sort's.  A run longer than BUCKET_BLOCK_MAX keys raises a flag,
// and the caller falls back to the radix sort.

constexpr uint32_t BUCKET_WARP_MAX = 512;     // runs up to this length: one warp (registers, then 4 KB of shared memory)
constexpr uint32_t BUCKET_BLOCK_MAX = 8192;   // longer runs up to this length: one block of 256, 64 KB
constexpr int BUCKET_WARPS = 8;

// keys of run nRuns (zero weight, outside the mesh) and any run index beyond it share the last bucket
__device__ __forceinline__ uint32_t bucket_run(uint64_t key, int pidBits, uint32_t nRuns) {
    const uint64_t r = key >> pidBits;
    return r < nRuns ? static_cast<uint32_t>(r) : nRuns;
}

// count[r] += keys in run r, r in [0, nRuns]; lanes of a warp with equal runs add once
__global__ void k_bucket_count(const uint64_t *keys, uint32_t n, int pidBits, uint32_t nRuns, uint32_t *count) {
    const unsigned lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t q = base + threadIdx.x;
        const bool ok = q < n;
        const uint32_t run = ok ? bucket_run(keys[q], pidBits, nRuns) : 0xFFFFFFFFu;
        const unsigned m = __match_any_sync(FULL, run);
        if (ok && static_cast<unsigned>(__ffs(m) - 1) == lane) atomicAdd(&count[run], static_cast<uint32_t>(__popc(m)));
    }
}

// The census weight of particle q for the sorted-weight array: from the key
// kernel's compact copy wc (8 bytes a particle, read back mostly from L2), or
// from the particle's record when there is none.
__device__ __forceinline__ double run_w(const Ctx &C, const CensusBank &cen, const double *wc, uint32_t q) {
    return wc ? wc[q] : census_w(C, cen, q);
}

// (key, q) to the next free slot of its run's range: cursor[r] starts at the run's first position.
// Each thread places PLACE_ILP keys per pass, their cursor atomics issued
// together, so that their round trips overlap.
constexpr int PLACE_ILP = 4;
__global__ void k_bucket_place(const uint64_t *keys, uint32_t n, int pidBits, uint32_t nRuns, uint32_t *cursor,
                               uint64_t *outKeys, uint32_t *outVals) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint64_t base = blockIdx.x * blockDim.x; base < n; base += static_cast<uint64_t>(PLACE_ILP) * stride) {
        uint32_t q[PLACE_ILP], run[PLACE_ILP], b[PLACE_ILP];
        uint64_t k[PLACE_ILP];
        unsigned m[PLACE_ILP];
#pragma unroll
        for (int u = 0; u < PLACE_ILP; ++u) {
            const uint64_t qq = base + static_cast<uint64_t>(u) * stride + threadIdx.x;
            q[u] = static_cast<uint32_t>(qq);
            k[u] = qq < n ? keys[qq] : 0ull;
            run[u] = qq < n ? bucket_run(k[u], pidBits, nRuns) : 0xFFFFFFFFu;
        }
#pragma unroll
        for (int u = 0; u < PLACE_ILP; ++u) {
            m[u] = __match_any_sync(FULL, run[u]);
            b[u] = 0;
            if (run[u] != 0xFFFFFFFFu && static_cast<int>(lane) == __ffs(m[u]) - 1)
                b[u] = atomicAdd(&cursor[run[u]], static_cast<uint32_t>(__popc(m[u])));
        }
#pragma unroll
        for (int u = 0; u < PLACE_ILP; ++u) {
            const uint32_t bb = __shfl_sync(FULL, b[u], __ffs(m[u]) - 1);
            if (run[u] != 0xFFFFFFFFu) {
                const uint32_t slot = bb + static_cast<uint32_t>(__popc(m[u] & lt));
                outKeys[slot] = k[u];
                outVals[slot] = q[u];
            }
        }
    }
}

// Ascending bitonic sort of s[0, P), P a power of two >= 2, by `threads`
// threads numbered t; `sync` orders the stages.  Each stage's pairs (i, i ^ j)
// are disjoint, and only the lower index of a pair touches it.
template <class Sync>
__device__ __forceinline__ void bitonic_sort(uint64_t *s, uint32_t P, uint32_t t, uint32_t threads, Sync sync) {
    for (uint32_t k = 2; k <= P; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = t; i < P; i += threads) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const uint64_t a = s[i], c = s[l];
                    if ((a > c) == ((i & k) == 0)) {
                        s[i] = c;
                        s[l] = a;
                    }
                }
            }
            sync();
        }
}

struct WarpSync {
    __device__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
    __device__ void operator()() const { __syncthreads(); }
};

// Within a run the key's run bits are fixed, so (hash << 32) | q orders the
// pairs by key; q < 2^32 - 1 and hash < 2^32 keep ~0 above every pair (padding).
__device__ __forceinline__ uint64_t bucket_pack(uint64_t key, uint32_t q, uint64_t hashMask) {
    return ((key & hashMask) << 32) | q;
}

// Ascending bitonic sort of 32 * E values held by a warp in registers, value
// e of lane l at index 32 e + l: stages with a distance of 32 or more pair a
// lane's own values, shorter ones pair lanes through shuffles.
template <int E>
__device__ __forceinline__ void warp_bitonic(uint64_t (&v)[E], uint32_t lane) {
    constexpr uint32_t P = 32u * E;
#pragma unroll
    for (uint32_t k = 2; k <= P; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const int d = static_cast<int>(j >> 5);
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int f = e ^ d;
                    if (f > e) {
                        const bool up = ((static_cast<uint32_t>(e) * 32u + lane) & k) == 0;
                        const uint64_t a = v[e], b = v[f];
                        if ((a > b) == up) {
                            v[e] = b;
                            v[f] = a;
                        }
                    }
                }
            } else {
                const bool lower = (lane & j) == 0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const uint64_t p = __shfl_xor_sync(FULL, static_cast<unsigned long long>(v[e]), static_cast<int>(j));
                    const bool up = ((static_cast<uint32_t>(e) * 32u + lane) & k) == 0;
                    const uint64_t lo = v[e] < p ? v[e] : p, hi = v[e] < p ? p : v[e];
                    v[e] = lower == up ? lo : hi;
                }
            }
        }
    }
}

// One run [b, b + len) with len <= 32 E, sorted by one warp in registers; the
// census weight of each sorted particle goes to wS.
template <int E>
__device__ __forceinline__ void warp_sort_run(const Ctx &C, const CensusBank &cen, uint64_t *keys, uint32_t *vals,
                                              double *wS, const double *wc, uint32_t b, uint32_t len, uint32_t r,
                                              int pidBits, uint64_t hashMask, uint32_t lane) {
    uint64_t v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint32_t i = static_cast<uint32_t>(e) * 32u + lane;
        v[e] = i < len ? bucket_pack(keys[b + i], vals[b + i], hashMask) : ~0ull;
    }
    warp_bitonic<E>(v, lane);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint32_t i = static_cast<uint32_t>(e) * 32u + lane;
        if (i < len) {
            const uint32_t q = static_cast<uint32_t>(v[e]);
            keys[b + i] = (static_cast<uint64_t>(r) << pidBits) | (v[e] >> 32);
            vals[b + i] = q;
            wS[b + i] = run_w(C, cen, wc, q);
        }
    }
}

// The same network on 32-bit words.
template <int E>
__device__ __forceinline__ void warp_bitonic32(uint32_t (&v)[E], uint32_t lane) {
    constexpr uint32_t P = 32u * E;
#pragma unroll
    for (uint32_t k = 2; k <= P; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const int d = static_cast<int>(j >> 5);
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int f = e ^ d;
                    if (f > e) {
                        const bool up = ((static_cast<uint32_t>(e) * 32u + lane) & k) == 0;
                        const uint32_t a = v[e], b = v[f];
                        if ((a > b) == up) {
                            v[e] = b;
                            v[f] = a;
                        }
                    }
                }
            } else {
                const bool lower = (lane & j) == 0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const uint32_t p = __shfl_xor_sync(FULL, v[e], static_cast<int>(j));
                    const bool up = ((static_cast<uint32_t>(e) * 32u + lane) & k) == 0;
                    const uint32_t lo = min(v[e], p), hi = max(v[e], p);
                    v[e] = lower == up ? lo : hi;
                }
            }
        }
    }
}

// A run of up to 32 E keys sorted as 32-bit words (hash << L) | position, when
// pidBits + L <= 31 (so every word is below the padding ~0): the hashes of a
// step's pids are distinct, so this is the order by key.  Each lane then takes
// its particle index from the lane and register that held that position.
template <int E>
__device__ __forceinline__ void warp_sort_run32(const Ctx &C, const CensusBank &cen, uint64_t *keys, uint32_t *vals,
                                                double *wS, const double *wc, uint32_t b, uint32_t len, uint32_t r,
                                                int pidBits, uint64_t hashMask, uint32_t lane) {
    constexpr uint32_t L = E == 1 ? 5u : (E == 2 ? 6u : 7u);
    uint32_t v[E], q0[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint32_t i = static_cast<uint32_t>(e) * 32u + lane;
        q0[e] = i < len ? vals[b + i] : 0u;
        v[e] = i < len ? (static_cast<uint32_t>(keys[b + i] & hashMask) << L) | i : ~0u;
    }
    warp_bitonic32<E>(v, lane);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint32_t i = static_cast<uint32_t>(e) * 32u + lane;
        const uint32_t pos = v[e] & ((1u << L) - 1u);
        uint32_t q = 0;
#pragma unroll
        for (int f = 0; f < E; ++f) {
            const uint32_t t = __shfl_sync(FULL, q0[f], static_cast<int>(pos & 31u));
            if ((pos >> 5) == static_cast<uint32_t>(f)) q = t;
        }
        if (i < len) {
            keys[b + i] = (static_cast<uint64_t>(r) << pidBits) | (v[e] >> L);
            vals[b + i] = q;
            wS[b + i] = run_w(C, cen, wc, q);
        }
    }
}

// Runs 0..nRuns-1 of (keys, vals), each sorted in place by key, with the census
// weights in sorted order to wS.  One warp per run of up to BUCKET_WARP_MAX
// keys: in registers up to 128 (fully unrolled networks; larger ones would not
// fit the instruction cache), in the warp's shared memory above.  Longer runs
// are listed for k_bucket_sort_long.
__global__ void __launch_bounds__(32 * BUCKET_WARPS) k_bucket_sort_runs(Ctx C, CensusBank cen, const double *wc,
                                                                        uint64_t *keys, uint32_t *vals, double *wS,
                                                                        const uint32_t *start, uint32_t nRuns,
                                                                        int pidBits, uint32_t *longRuns,
                                                                        uint32_t *nLong, uint32_t longCap) {
    __shared__ uint64_t sm[BUCKET_WARPS][BUCKET_WARP_MAX];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t *sw = sm[wid];
    const uint64_t hashMask = (1ull << pidBits) - 1ull;   // pidBits <= 32
    const uint32_t warps = gridDim.x * BUCKET_WARPS;
    for (uint32_t r = blockIdx.x * BUCKET_WARPS + wid; r < nRuns; r += warps) {
        const uint32_t b = start[r], len = start[r + 1] - b;
        if (len == 0) continue;
        if (len == 1) {
            if (lane == 0) wS[b] = run_w(C, cen, wc, vals[b]);
        } else if (len <= 32) {
            if (pidBits <= 26) warp_sort_run32<1>(C, cen, keys, vals, wS, wc, b, len, r, pidBits, hashMask, lane);
            else warp_sort_run<1>(C, cen, keys, vals, wS, wc, b, len, r, pidBits, hashMask, lane);
        } else if (len <= 64) {
            if (pidBits <= 25) warp_sort_run32<2>(C, cen, keys, vals, wS, wc, b, len, r, pidBits, hashMask, lane);
            else warp_sort_run<2>(C, cen, keys, vals, wS, wc, b, len, r, pidBits, hashMask, lane);
        } else if (len <= 128) {
            if (pidBits <= 24) warp_sort_run32<4>(C, cen, keys, vals, wS, wc, b, len, r, pidBits, hashMask, lane);
            else warp_sort_run<4>(C, cen, keys, vals, wS, wc, b, len, r, pidBits, hashMask, lane);
        } else if (len <= BUCKET_WARP_MAX) {
            uint32_t P = 256;
            while (P < len) P <<= 1;
            for (uint32_t i = lane; i < P; i += 32)
                sw[i] = i < len ? bucket_pack(keys[b + i], vals[b + i], hashMask) : ~0ull;
            __syncwarp();
            bitonic_sort(sw, P, lane, 32u, WarpSync{});
            for (uint32_t i = lane; i < len; i += 32) {
                const uint64_t v = sw[i];
                const uint32_t q = static_cast<uint32_t>(v);
                keys[b + i] = (static_cast<uint64_t>(r) << pidBits) | (v >> 32);
                vals[b + i] = q;
                wS[b + i] = run_w(C, cen, wc, q);
            }
            __syncwarp();
        } else if (lane == 0) {
            const uint32_t slot = atomicAdd(nLong, 1u);
            if (slot < longCap) longRuns[slot] = r;
        }
    }
}

// The listed runs, one block each (dynamic shared memory: BUCKET_BLOCK_MAX words).
// A run longer than BUCKET_BLOCK_MAX, or more listed runs than longCap, sets *tooLong.
__global__ void __launch_bounds__(256) k_bucket_sort_long(Ctx C, CensusBank cen, const double *wc, uint64_t *keys,
                                                          uint32_t *vals,
                                                          double *wS, const uint32_t *start, int pidBits,
                                                          const uint32_t *longRuns, const uint32_t *nLong,
                                                          uint32_t longCap, uint32_t *tooLong) {
    extern __shared__ __align__(16) unsigned char bucketMem[];
    uint64_t *sb = reinterpret_cast<uint64_t *>(bucketMem);
    const uint32_t listed = *nLong;
    if (listed > longCap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *tooLong = 1u;
        return;
    }
    const uint64_t hashMask = (1ull << pidBits) - 1ull;
    for (uint32_t e = blockIdx.x; e < listed; e += gridDim.x) {
        const uint32_t r = longRuns[e];
        const uint32_t b = start[r], len = start[r + 1] - b;
        if (len > BUCKET_BLOCK_MAX) {
            if (threadIdx.x == 0) *tooLong = 1u;
            continue;
        }
        uint32_t P = 32;
        while (P < len) P <<= 1;
        for (uint32_t i = threadIdx.x; i < P; i += blockDim.x)
            sb[i] = i < len ? bucket_pack(keys[b + i], vals[b + i], hashMask) : ~0ull;
        __syncthreads();
        bitonic_sort(sb, P, threadIdx.x, blockDim.x, BlockSync{});
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
            const uint64_t v = sb[i];
            const uint32_t q = static_cast<uint32_t>(v);
            keys[b + i] = (static_cast<uint64_t>(r) << pidBits) | (v >> 32);
            vals[b + i] = q;
            wS[b + i] = run_w(C, cen, wc, q);
        }
        __syncthreads();
    }
}

// first sorted position of each cell (lower_bound of cell << pidBits), cells 0..N
__global__ void k_comb_ranges(const uint64_t *keys, uint32_t n, uint32_t ncells, uint32_t *start, int pidBits) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncells; c += gridDim.x * blockDim.x) {
        const uint64_t v = static_cast<uint64_t>(c) << pidBits;
        uint32_t first = 0, count = n;
        while (count > 0) {
            uint32_t step = count >> 1, it = first + step;
            if (keys[it] < v) { first = it + 1; count -= step + 1; } else count = step;
        }
        start[c] = first;
    }
}

// census weights in sorted order (one gather, so the per-cell loops read contiguous memory)
__global__ void k_sorted_weights(Ctx C, CensusBank cen, const uint32_t *idx, uint32_t n, double *wS) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        wS[q] = census_w(C, cen, idx[q]);
}

// weights[cell] (:136-141), summed in sorted order
__global__ void k_comb_cell_sums(const double *wS, const uint32_t *start, uint32_t ncells, double *W) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint32_t q = start[c]; q < start[c + 1]; ++q) s += wS[q];
        W[c] = s;
    }
}

// Deterministic total: thread t adds v[t], v[t + 1024], ... in order (coalesced),
// then a pairwise tree over the 1024 partial sums.
__global__ void k_blocked_sum(const double *v, uint32_t n, double *out) {
    __shared__ double part[1024];
    double s = 0.0;
    for (uint32_t q = threadIdx.x; q < n; q += 1024) s += v[q];
    part[threadIdx.x] = s;
    __syncthreads();
    for (uint32_t w = 512; w >= 1; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] = part[threadIdx.x] + part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

struct CombCell {
    uint64_t nin;
    double w_ideal;   // split path
    double e;         // comb path: new_energy
    double r;
    int mode;         // 0 keep/split, 1 comb
};

__device__ __forceinline__ CombCell comb_cell_params(const Ctx &C, const CombParams &P, uint32_t c, uint32_t cnt,
                                                     double Wc, double Wtot) {
    CombCell cc;
    uint64_t share = static_cast<uint64_t>(static_cast<double>(P.ntotal) * Wc / Wtot);
    uint64_t lo = share > P.nmin ? share : P.nmin;
    cc.nin = (P.nmin * 20 < lo) ? P.nmin * 20 : lo;
    cc.mode = (cnt <= cc.nin) ? 0 : 1;
    cc.w_ideal = Wc / static_cast<double>(cc.nin);
    cc.e = cc.w_ideal;
    cc.r = cc.mode ? stream_uniform(C.seedLo, C.seedHi, TAG_COMB, C.step, c, 0) : 0.0;
    return cc;
}

// Per cell (:161-226): the number of copies of each sorted particle, the weight
// of those copies, and the cell's census radiation energy summed in output order
// (RadiationIMC::postStep :2013-2016).  pCount bit 31 marks a particle kept as is.
constexpr uint32_t KEEP = 0x80000000u;
__global__ void k_comb_plan(Ctx C, CombParams P, const double *wS, const uint32_t *start, const double *W,
                            const double *Wtot, uint32_t *pCount, double *pWeight, uint64_t *cellCount,
                            double *eradCensus, DevStats *st) {
    const double tot = *Wtot;
    if (!isfinite(tot)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(C, STORM_DERR_COMB_TOTAL, 0, 0);
    }
    double eOut = 0.0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        const uint32_t a = start[c], b = start[c + 1];
        double ecell = 0.0;
        uint64_t m = 0;
        if (tot == 0.0 || !isfinite(tot) || a == b) {
            for (uint32_t q = a; q < b; ++q) pCount[q] = 0;
        } else {
            CombCell cc = comb_cell_params(C, P, c, b - a, W[c], tot);
            if (cc.mode == 0) {
                for (uint32_t q = a; q < b; ++q) {
                    const double w = wS[q];
                    if (w > 2 * cc.w_ideal) {
                        const uint64_t ns = static_cast<uint64_t>(ceil(w / cc.w_ideal));
                        const double ws = w / static_cast<double>(ns);
                        for (uint64_t k = 0; k < ns; ++k) ecell += ws;
                        pCount[q] = static_cast<uint32_t>(ns);
                        pWeight[q] = ws;
                        m += ns;
                    } else {
                        ecell += w;
                        pCount[q] = 1u | KEEP;
                        pWeight[q] = w;
                        m += 1;
                    }
                }
            } else {
                uint64_t k = 0;
                double cum = 0;
                for (uint32_t q = a; q < b; ++q) {
                    const double w = wS[q];
                    const uint64_t k0 = k;
                    while ((cum + w) > (static_cast<double>(k) + cc.r) * cc.e) {
                        ++k;
                        ecell += cc.e;
                    }
                    cum += w;
                    pCount[q] = static_cast<uint32_t>(k - k0);
                    pWeight[q] = cc.e;
                }
                m = k;
            }
        }
        cellCount[c] = m;
        eradCensus[c] = ecell;
        eOut += ecell;
    }
    eOut = warp_sum(eOut);
    if ((threadIdx.x & 31) == 0 && eOut != 0.0) atomicAdd(&st->eCensusOut, eOut);
}

// #{k >= 0 : (k + r) E < P}: the comb index a sequential walk holds once it
// has passed weight P (the loop condition of :203-222 with cum = P).
__device__ __forceinline__ uint64_t teeth_below(double P, double r, double E) {
    if (!(P > 0.0)) return 0;
    const double g = P / E - r;
    uint64_t k = g > 0.0 ? static_cast<uint64_t>(ceil(g)) : 0;
    while (k > 0 && (static_cast<double>(k - 1) + r) * E >= P) --k;
    while ((static_cast<double>(k) + r) * E < P) ++k;
    return k;
}

// Exchange 2 of a sharded comb: every (shard, cell) run's weight and particle
// count, this handle's runs filled and the others zero, as doubles.
__global__ void k_shard_pack_runs(const double *runW, const uint32_t *start, uint32_t nRuns, double *x) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nRuns; r += gridDim.x * blockDim.x) {
        x[r] = runW[r];
        x[nRuns + r] = static_cast<double>(start[r + 1] - start[r]);
    }
}

// A cell's global weight: its runs' weights added in shard order (every
// handle adds the same numbers in the same order).
__global__ void k_shard_cell_weights(const double *x, uint32_t ncells, uint32_t shards, double *Wc) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
        double w = 0.0;
        for (uint32_t sh = 0; sh < shards; ++sh) w += x[static_cast<size_t>(sh) * ncells + c];
        Wc[c] = w;
    }
}

// CombPopulationControl::activate's plan over particle shards.  x holds every
// run's weight (S N) and count (S N) after exchange 2; Wc the cells' global
// weights.  A cell's targets come from its global weight and count; a combed
// cell's teeth run along its runs in shard order, run s starting at the
// weight P of the runs below it and at comb index teeth_below(P).  Only this
// handle's shards [lo, hi) hold particles here.  eradCensus gets this
// handle's part of each cell's census energy.
__global__ void k_comb_plan_sharded(Ctx C, CombParams P, const double *wS, const uint32_t *start, const double *x,
                                    const double *Wc, const double *Wtot, uint32_t lo, uint32_t hi,
                                    uint32_t *pCount, double *pWeight, double *eradCensus, DevStats *st) {
    const double tot = *Wtot;
    if (!isfinite(tot)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(C, STORM_DERR_COMB_TOTAL, 0, 0);
    }
    const uint32_t N = C.ncells, S = C.shards;
    const size_t R = static_cast<size_t>(S) * N;
    double eOut = 0.0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        uint64_t cnt = 0;
        for (uint32_t sh = 0; sh < S; ++sh) cnt += static_cast<uint64_t>(x[R + static_cast<size_t>(sh) * N + c]);
        double ecell = 0.0;
        const bool none = tot == 0.0 || !isfinite(tot) || cnt == 0;
        const CombCell cc = none ? CombCell{} : comb_cell_params(C, P, c, static_cast<uint32_t>(cnt), Wc[c], tot);
        double below = 0.0;   // weight of this cell's runs in the shards before sh
        for (uint32_t sh = 0; sh < hi; ++sh) {
            const size_t run = static_cast<size_t>(sh) * N + c;
            if (sh < lo) {
                below += x[run];
                continue;
            }
            const uint32_t a = start[run], b = start[run + 1];
            if (none) {
                for (uint32_t q = a; q < b; ++q) pCount[q] = 0;
            } else if (cc.mode == 0) {
                for (uint32_t q = a; q < b; ++q) {
                    const double w = wS[q];
                    if (w > 2 * cc.w_ideal) {
                        const uint64_t ns = static_cast<uint64_t>(ceil(w / cc.w_ideal));
                        const double ws = w / static_cast<double>(ns);
                        for (uint64_t k = 0; k < ns; ++k) ecell += ws;
                        pCount[q] = static_cast<uint32_t>(ns);
                        pWeight[q] = ws;
                    } else {
                        ecell += w;
                        pCount[q] = 1u | KEEP;
                        pWeight[q] = w;
                    }
                }
            } else {
                double cum = below;
                uint64_t k = teeth_below(cum, cc.r, cc.e);
                for (uint32_t q = a; q < b; ++q) {
                    const double w = wS[q];
                    const uint64_t k0 = k;
                    while ((cum + w) > (static_cast<double>(k) + cc.r) * cc.e) {
                        ++k;
                        ecell += cc.e;
                    }
                    cum += w;
                    pCount[q] = static_cast<uint32_t>(k - k0);
                    pWeight[q] = cc.e;
                }
            }
            below += x[run];
        }
        eradCensus[c] = ecell;
        eOut += ecell;
    }
    eOut = warp_sum(eOut);
    if ((threadIdx.x & 31) == 0 && eOut != 0.0) atomicAdd(&st->eCensusOut, eOut);
}

// Exchange 3 of a sharded comb: this handle's census particles per shard (the
// copies its runs of shard s produce: the exclusive scan of the copy counts at
// the shard's run boundaries) and its part of each cell's census energy.
__global__ void k_shard_pack_census(const uint64_t *pOff, const uint64_t *total, const uint32_t *start, uint32_t n,
                                    uint32_t ncells, uint32_t shards, uint32_t lo, uint32_t hi,
                                    const double *eradCensus, double *x) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < shards) {
        double v = 0.0;
        if (t >= lo && t < hi) {
            const uint32_t a = start[static_cast<size_t>(t) * ncells], b = start[static_cast<size_t>(t + 1) * ncells];
            const uint64_t oa = a < n ? pOff[a] : *total, ob = b < n ? pOff[b] : *total;
            v = static_cast<double>(ob - oa);
        }
        x[t] = v;
    }
    for (uint32_t c = t; c < ncells; c += gridDim.x * blockDim.x) x[shards + c] = eradCensus[c];
}

// y[i] += x[i]
__global__ void k_add_into(double *y, const double *x, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += x[i];
}

// One thread per sorted particle writes its copies at its output offset.
// The exclusive prefix of the copy counts over sorted particles is the output
// position: cells are contiguous in sorted order and the output is cell-major.
// Each thread takes EMIT_BATCH sorted particles per iteration and issues all
// of their census-record gathers (read-only loads) before it writes any copy,
// so the random reads overlap.
constexpr int EMIT_BATCH = 2;

// The copy of a census particle the comb writes (FP64 form): the new weight
// unless kept, and a position outside the box pulled toward the cell centre.
__device__ __forceinline__ void comb_copy_fp64(const Ctx &C, PartReg &p, uint32_t c, uint32_t raw, double wNew) {
    if (!(raw & KEEP)) { p.w = wNew; p.w0 = p.w; p.t = 0; }
    p.cell = c;
    if (outside_box(C, p.x, p.y, p.z)) {   // :228-250
        double mx, my, mz;
        mesh_point(C, c, mx, my, mz);
        const double ox = p.x, oy = p.y, oz = p.z, dx = mx - ox, dy = my - oy, dz = mz - oz;
        double t = 1e-6;
        while (outside_box(C, p.x, p.y, p.z) && t < 1.0) {
            p.x = ox + t * dx; p.y = oy + t * dy; p.z = oz + t * dz;
            t *= 2;
        }
        if (outside_box(C, p.x, p.y, p.z)) { p.x = mx; p.y = my; p.z = mz; }
    }
}
__device__ __forceinline__ void comb_emit_fp64(const Ctx &C, PartReg &p, uint32_t c, uint32_t raw, double wNew,
                                               uint64_t o, const Bank &out) {
    comb_copy_fp64(C, p, c, raw, wNew);
    const uint32_t m = raw & ~KEEP;
    for (uint32_t k = 0; k < m; ++k) store_part(out, static_cast<uint32_t>(o + k), p, static_cast<uint32_t>(o + k), 0);
}

template <bool FP32>
__global__ void k_comb_emit(Ctx C, CensusBank cen, const uint32_t *idx, const uint64_t *sortedKeys, int pidBits,
                            uint32_t bins, uint32_t nValid, const uint32_t *pCount, const double *pWeight,
                            const uint64_t *pOffset, Bank out) {
    const uint32_t stride = gridDim.x * blockDim.x;
    constexpr int words = FP32 ? 4 : 6;
    for (uint32_t base = blockIdx.x * blockDim.x + threadIdx.x; base < nValid; base += EMIT_BATCH * stride) {
        uint32_t raw[EMIT_BATCH], src[EMIT_BATCH];
        uint4 rec[EMIT_BATCH][words];
#pragma unroll
        for (int u = 0; u < EMIT_BATCH; ++u) {
            const uint32_t q = base + u * stride;
            raw[u] = q < nValid ? pCount[q] : 0u;
            src[u] = (raw[u] & ~KEEP) ? idx[q] : 0u;
        }
#pragma unroll
        for (int u = 0; u < EMIT_BATCH; ++u) {
            if (raw[u] & ~KEEP) {
                const uint4 *r = cen.rec + static_cast<size_t>(src[u]) * words;
#pragma unroll
                for (int w = 0; w < words; ++w) rec[u][w] = __ldg(r + w);
            }
        }
#pragma unroll
        for (int u = 0; u < EMIT_BATCH; ++u) {
            const uint32_t m = raw[u] & ~KEEP;
            if (m == 0) continue;
            const uint32_t q = base + u * stride;
            const uint32_t c = cell_of_run(C, sortedKeys[q] >> pidBits, bins);
            const uint64_t o = pOffset[q];
            const double wNew = pWeight[q];
            if constexpr (FP32) {
                const uint4 a = rec[u][0], b = rec[u][1], d = rec[u][2];
                Track32 T;
                T.qx = __uint_as_float(a.x); T.qy = __uint_as_float(a.y); T.qz = __uint_as_float(a.z);
                T.ux = __uint_as_float(a.w); T.uy = __uint_as_float(b.x); T.uz = __uint_as_float(b.y);
                T.t = __longlong_as_double((static_cast<unsigned long long>(b.w) << 32) | b.z);
                T.w = lo_double(d); T.w0 = hi_double(d);
                if (!(raw[u] & KEEP)) { T.w = wNew; T.w0 = T.w; T.t = 0; }
                T.cell = c;
                const float nu = __uint_as_float(rec[u][3].w);
                for (uint32_t k = 0; k < m; ++k) {
                    store32(out, static_cast<uint32_t>(o + k), T, static_cast<uint32_t>(o + k), 0);
                    if (out.nu) store_nu32(out, static_cast<uint32_t>(o + k), nu);
                }
            } else {
                const uint4 a = rec[u][0], b = rec[u][1], d = rec[u][2], e = rec[u][3], f = rec[u][4];
                PartReg p;
                p.x = lo_double(a); p.y = hi_double(a);
                p.z = lo_double(b); p.vx = hi_double(b);
                p.vy = lo_double(d); p.vz = hi_double(d);
                p.t = lo_double(e); p.w = hi_double(e);
                p.w0 = lo_double(f);
                p.nu = hi_double(rec[u][5]);
                comb_emit_fp64(C, p, c, raw[u], wNew, o, out);
            }
        }
    }
}

// Output-driven form of the same write: one thread per output slot o, whose
// source is the sorted particle src[o].  Every lane writes one particle, so
// the bank writes are contiguous and no lane idles on a dropped particle.
// src[o] comes from marking each particle with copies at its first slot and a
// running maximum over the slots (the sources increase with the slots).
__global__ void k_emit_src_mark(const uint32_t *pCount, const uint64_t *pOffset, uint32_t nValid, uint32_t *src) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nValid; q += gridDim.x * blockDim.x)
        if (pCount[q] & ~KEEP) src[pOffset[q]] = q;
}

// inclusive running maximum of v[0, n) in tiles of 1024 (the tile's maximum to tileMax)
__global__ void __launch_bounds__(1024) k_max_tiles(uint32_t *v, uint32_t n, uint32_t *tileMax) {
    __shared__ uint32_t wmax[32];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t q = blockIdx.x * 1024u + threadIdx.x;
    uint32_t x = q < n ? v[q] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, d);
        if (static_cast<int>(lane) >= d) x = max(x, y);
    }
    if (lane == 31) wmax[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = wmax[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, w, d);
            if (static_cast<int>(lane) >= d) w = max(w, y);
        }
        wmax[lane] = w;
    }
    __syncthreads();
    if (wid > 0) x = max(x, wmax[wid - 1]);
    if (q < n) v[q] = x;
    if (threadIdx.x == 1023) tileMax[blockIdx.x] = x;
}
// tileMax[t] <- maximum of tiles 0..t-1 (0 for t = 0), one block
__global__ void __launch_bounds__(1024) k_max_tile_prefix(uint32_t *tileMax, uint32_t ntiles) {
    __shared__ uint32_t wmax[32];
    __shared__ uint32_t carryS;
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < ntiles; base += 1024u) {
        const uint32_t q = base + threadIdx.x;
        uint32_t x = q < ntiles ? tileMax[q] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, x, d);
            if (static_cast<int>(lane) >= d) x = max(x, y);
        }
        if (lane == 31) wmax[wid] = x;
        __syncthreads();
        if (wid == 0) {
            uint32_t w = wmax[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, w, d);
                if (static_cast<int>(lane) >= d) w = max(w, y);
            }
            wmax[lane] = w;
        }
        __syncthreads();
        if (wid > 0) x = max(x, wmax[wid - 1]);
        const uint32_t incl = max(x, carry);
        // exclusive: the inclusive maximum of the previous entry
        uint32_t prev = __shfl_up_sync(FULL, incl, 1);
        if (lane == 0) prev = wid > 0 ? max(wmax[wid - 1], carry) : carry;
        if (q < ntiles) tileMax[q] = prev;
        if (threadIdx.x == 1023) carryS = incl;
        __syncthreads();
        carry = carryS;
        __syncthreads();
    }
}
__global__ void __launch_bounds__(1024) k_max_apply(uint32_t *v, uint32_t n, const uint32_t *tileMax) {
    const uint32_t q = blockIdx.x * 1024u + threadIdx.x;
    if (q < n) v[q] = max(v[q], tileMax[blockIdx.x]);
}

template <bool FP32>
__global__ void k_comb_emit_out(Ctx C, CensusBank cen, const uint32_t *idx, const uint64_t *sortedKeys, int pidBits,
                                uint32_t bins, uint32_t total, const uint32_t *src, const uint32_t *pCount,
                                const double *pWeight, Bank out) {
    constexpr int words = FP32 ? 4 : 6;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + threadIdx.x; base < total; base += EMIT_BATCH * stride) {
        uint32_t qs[EMIT_BATCH], raw[EMIT_BATCH];
        uint4 rec[EMIT_BATCH][words];
#pragma unroll
        for (int u = 0; u < EMIT_BATCH; ++u) {
            const uint32_t o = base + u * stride;
            qs[u] = o < total ? src[o] : 0u;
        }
#pragma unroll
        for (int u = 0; u < EMIT_BATCH; ++u) {
            const uint32_t o = base + u * stride;
            raw[u] = 0u;
            if (o < total) {
                raw[u] = pCount[qs[u]];
                const uint4 *r = cen.rec + static_cast<size_t>(idx[qs[u]]) * words;
#pragma unroll
                for (int w = 0; w < words; ++w) rec[u][w] = __ldg(r + w);
            }
        }
#pragma unroll
        for (int u = 0; u < EMIT_BATCH; ++u) {
            const uint32_t o = base + u * stride;
            if (o >= total) continue;
            const uint32_t q = qs[u];
            const uint32_t c = cell_of_run(C, sortedKeys[q] >> pidBits, bins);
            const double wNew = pWeight[q];
            if constexpr (FP32) {
                const uint4 a = rec[u][0], b = rec[u][1], d = rec[u][2];
                Track32 T;
                T.qx = __uint_as_float(a.x); T.qy = __uint_as_float(a.y); T.qz = __uint_as_float(a.z);
                T.ux = __uint_as_float(a.w); T.uy = __uint_as_float(b.x); T.uz = __uint_as_float(b.y);
                T.t = __longlong_as_double((static_cast<unsigned long long>(b.w) << 32) | b.z);
                T.w = lo_double(d); T.w0 = hi_double(d);
                if (!(raw[u] & KEEP)) { T.w = wNew; T.w0 = T.w; T.t = 0; }
                T.cell = c;
                store32(out, o, T, o, 0);
                if (out.nu) store_nu32(out, o, __uint_as_float(rec[u][3].w));
            } else {
                const uint4 a = rec[u][0], b = rec[u][1], d = rec[u][2], e = rec[u][3], f = rec[u][4];
                PartReg p;
                p.x = lo_double(a); p.y = hi_double(a);
                p.z = lo_double(b); p.vx = hi_double(b);
                p.vy = lo_double(d); p.vz = hi_double(d);
                p.t = lo_double(e); p.w = hi_double(e);
                p.w0 = lo_double(f);
                p.nu = hi_double(rec[u][5]);
                comb_copy_fp64(C, p, c, raw[u], wNew);
                store_part(out, o, p, o, 0);
            }
        }
    }
}

// ------------------------------------------------------------------ stratified comb
// StratifiedCombPopulationControl::activate (population/CombPopulationControl.hpp:255-511)
// with its classifier lowered to frequency bins.  The census is sorted by
// (cell, bin, keyed hash of pid), so each (cell, bin) is one contiguous run in
// a pseudo-random order (the reference's sort by id and shuffle); per cell the
// bin targets follow the reference's allocation, and each bin is kept, split
// or combed like appendCombBin.

// the census particle's photon energy
__device__ __forceinline__ double census_nu(const Ctx &C, const CensusBank &c, uint32_t q) {
    if (C.fp32) return static_cast<double>(__uint_as_float(c.rec[static_cast<size_t>(q) * 4 + 3].w));
    return hi_double(c.rec[static_cast<size_t>(q) * 6 + 5]);
}
// the bin of frequency nu: the first g with nu < bounds[g + 1], else the last
// (RadiationOpacityModel::findGroup's rule, radiation/RadiationOpacityModel.hpp:76-86)
__device__ __forceinline__ uint32_t strat_bin(const StratParams &S, double nu) {
    if (S.bins <= 1) return 0;
    uint32_t lo = 0, hi = S.bins - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (nu < S.bounds[mid + 1]) hi = mid; else lo = mid + 1;
    }
    return lo;
}

__global__ void k_strat_keys(Ctx C, CensusBank cen, uint32_t n, uint64_t *keys, uint32_t *vals, uint32_t combKey,
                             int pidBits, StratParams S, double *wc) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const double w = census_w(C, cen, q);
        if (wc) wc[q] = w;
        const uint2 cp = census_cell_pid(C, cen, q);
        const uint32_t pid = cp.y;
        uint32_t cell = cp.x;
        if (!C.fp32) {   // :288-295
            const uint4 a = cen.rec[static_cast<size_t>(q) * 6], b = cen.rec[static_cast<size_t>(q) * 6 + 1];
            if (outside_box(C, lo_double(a), hi_double(a), lo_double(b))) raise_error(C, STORM_DERR_COMB_OUTSIDE, cell, pid);
        }
        const bool badWeight = !isfinite(w) || w < 0.0;   // :296-309
        if (badWeight) raise_error(C, STORM_DERR_COMB_WEIGHT, cell, pid);
        uint64_t cb;
        if (w == 0.0 || badWeight || cell >= C.ncells) cb = static_cast<uint64_t>(C.ncells) * S.bins;   // :310-311
        else cb = static_cast<uint64_t>(cell) * S.bins + strat_bin(S, census_nu(C, cen, q));
        keys[q] = (cb << pidBits) | comb_hash(pid, combKey, pidBits);
        vals[q] = q;
    }
}

// binWeights[cell][g] and cellWeights[cell] (:326-328), summed in sorted order
__global__ void k_strat_sums(const double *wS, const uint32_t *start, uint32_t ncells, uint32_t bins, double *binW,
                             double *cellW) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
        double cs = 0.0;
        for (uint32_t g = 0; g < bins; ++g) {
            const size_t cb = static_cast<size_t>(c) * bins + g;
            double s = 0.0;
            for (uint32_t q = start[cb]; q < start[cb + 1]; ++q) s += wS[q];
            binW[cb] = s;
            cs += s;
        }
        cellW[c] = cs;
    }
}

// Per cell (:416-488): the cell's target, each bin's share of it, then each
// bin as appendCombBin (:347-413) writes it: copy counts and weights of the
// sorted particles (bit 31 of the count: kept as is) and the census energy.
__global__ void k_strat_plan(Ctx C, CombParams P, StratParams S, const double *wS, const uint32_t *start,
                             const double *binW, const double *cellW, const double *Wtot, uint32_t *pCount,
                             double *pWeight, uint64_t *cellCount, double *eradCensus, DevStats *st) {
    const double tot = *Wtot;
    if (!isfinite(tot)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(C, STORM_DERR_COMB_TOTAL, 0, 0);
    }
    const uint32_t B = S.bins;
    double eOut = 0.0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        const size_t base = static_cast<size_t>(c) * B;
        const uint32_t a0 = start[base], aEnd = start[base + B];
        const double cw = cellW[c];
        double ecell = 0.0;
        uint64_t m = 0;
        if (tot == 0.0 || !isfinite(tot) || !(cw > 0.0) || a0 == aEnd) {
            for (uint32_t q = a0; q < aEnd; ++q) pCount[q] = 0;
        } else {
            const uint64_t share = static_cast<uint64_t>(static_cast<double>(P.ntotal) * cw / tot);
            const uint64_t lo = share > P.nmin ? share : P.nmin;
            const uint64_t cellTarget = (P.nmin * 20 < lo) ? P.nmin * 20 : lo;
            uint8_t act[STORM_STRAT_MAX_BINS];
            uint64_t target[STORM_STRAT_MAX_BINS];
            double frac[STORM_STRAT_MAX_BINS];
            uint32_t nAct = 0;
            for (uint32_t g = 0; g < B; ++g) {
                target[g] = 0;
                frac[g] = 0.0;
                if (start[base + g + 1] > start[base + g]) act[nAct++] = static_cast<uint8_t>(g);
            }
            uint64_t allocated = 0;
            if (static_cast<uint64_t>(nAct) * S.minPerBin <= cellTarget) {
                for (uint32_t a = 0; a < nAct; ++a) { target[act[a]] = S.minPerBin; allocated += S.minPerBin; }
            } else {
                // heaviest bins first (ties keep ascending bin order)
                for (uint32_t a = 1; a < nAct; ++a) {
                    const uint8_t g = act[a];
                    uint32_t b = a;
                    while (b > 0 && binW[base + act[b - 1]] < binW[base + g]) { act[b] = act[b - 1]; --b; }
                    act[b] = g;
                }
                const uint64_t prot = nAct < cellTarget ? nAct : cellTarget;
                for (uint64_t a = 0; a < prot; ++a) { target[act[a]] = 1; ++allocated; }
            }
            const uint64_t remaining = cellTarget > allocated ? cellTarget - allocated : 0;
            uint64_t prop = 0;
            for (uint32_t a = 0; a < nAct; ++a) {
                const uint32_t g = act[a];
                if (target[g] == 0) continue;
                const double exact = static_cast<double>(remaining) * binW[base + g] / cw;
                const uint64_t extra = static_cast<uint64_t>(floor(exact));
                target[g] += extra;
                prop += extra;
                frac[g] = exact - static_cast<double>(extra);
            }
            while (prop < remaining) {
                uint32_t best = B;
                double bf = -1.0;
                for (uint32_t a = 0; a < nAct; ++a) {
                    const uint32_t g = act[a];
                    if (target[g] > 0 && frac[g] > bf) { best = g; bf = frac[g]; }
                }
                if (best == B) break;
                ++target[best];
                frac[best] = 0.0;
                ++prop;
            }
            for (uint32_t g = 0; g < B; ++g) {
                const uint32_t a = start[base + g], b = start[base + g + 1];
                const double bw = binW[base + g];
                const uint64_t tg = target[g];
                if (a == b) continue;
                if (tg == 0 || !(bw > 0.0)) {   // a bin without a target loses its particles (:349-350)
                    for (uint32_t q = a; q < b; ++q) pCount[q] = 0;
                } else if (static_cast<uint64_t>(b - a) <= tg) {
                    const double ideal = bw / static_cast<double>(tg);
                    for (uint32_t q = a; q < b; ++q) {
                        const double w = wS[q];
                        if (w > 2.0 * ideal) {
                            const uint64_t ns = static_cast<uint64_t>(ceil(w / ideal));
                            const double ws = w / static_cast<double>(ns);
                            for (uint64_t k = 0; k < ns; ++k) ecell += ws;
                            pCount[q] = static_cast<uint32_t>(ns);
                            pWeight[q] = ws;
                            m += ns;
                        } else {
                            ecell += w;
                            pCount[q] = 1u | KEEP;
                            pWeight[q] = w;
                            m += 1;
                        }
                    }
                } else {
                    const double newWeight = bw / static_cast<double>(tg);
                    const double r = stream_uniform(C.seedLo, C.seedHi, TAG_COMB, C.step, c, 1 + g);
                    uint64_t k = 0;
                    double cum = 0.0;
                    for (uint32_t q = a; q < b; ++q) {
                        const double w = wS[q];
                        const uint64_t k0 = k;
                        while ((cum + w) > (static_cast<double>(k) + r) * newWeight && k < tg) {
                            ++k;
                            ecell += newWeight;
                        }
                        cum += w;
                        pCount[q] = static_cast<uint32_t>(k - k0);
                        pWeight[q] = newWeight;
                    }
                    m += k;
                }
            }
        }
        cellCount[c] = m;
        eradCensus[c] = ecell;
        eOut += ecell;
    }
    eOut = warp_sum(eOut);
    if ((threadIdx.x & 31) == 0 && eOut != 0.0) atomicAdd(&st->eCensusOut, eOut);
}

// copies per sorted slot, over n slots of which the first *nValid are particles (zero beyond)
__global__ void k_mask_count_upto(const uint32_t *pCount, uint32_t n, const uint32_t *nValid, uint64_t *out) {
    const uint32_t v = *nValid;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        out[q] = q < v ? (pCount[q] & ~KEEP) : 0ull;
}

// census kept as is (no population control): order by pid for a deterministic bank
__global__ void k_census_keys_pid(Ctx C, CensusBank cen, uint32_t n, uint64_t *keys, uint32_t *vals) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        keys[q] = census_cell_pid(C, cen, q).y;
        vals[q] = q;
    }
}
__global__ void k_gather(Ctx C, CensusBank src, const uint32_t *idx, uint32_t n, Bank dst, double *eradCensus,
                         DevStats *st) {
    double e = 0.0;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t sq = idx[q];
        double w;
        uint32_t cell, pid_, draw_;
        if (C.fp32) {
            Track32 T;
            census_load32(src, sq, T, pid_, draw_);
            store32(dst, q, T, q, 0);
            if (dst.nu) store_nu32(dst, q, T.nu);
            w = T.w; cell = T.cell;
        } else {
            PartReg p;
            census_load64(src, sq, p, pid_, draw_);
            store_part(dst, q, p, q, 0);
            w = p.w; cell = p.cell;
        }
        atomicAdd(eradCensus + cell, w);
        e += w;
    }
    e = warp_sum(e);
    if ((threadIdx.x & 31) == 0 && e != 0.0) atomicAdd(&st->eCensusOut, e);
}

// ------------------------------------------------------------------ poststep
// RadiationIMC::postStep (radiation/RadiationIMC.hpp:1887-2029), gray, no hydro.
__global__ void k_poststep(Ctx C, CellArrays A, OpacityEos M, double dt) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C.ncells; c += gridDim.x * blockDim.x) {
        if (C.fixMat) {   // reproducible tallies: fold the fixed-point sums of the transport
            A.eint[c] += fixed_value(C.fixMat, c) * (1.0 / C.fixScaleMat);
            A.eradAvg[c] += fixed_value(C.fixRad, c) * (1.0 / C.fixScaleRad);
        }
        A.eradAvg[c] /= (dt * A.vol[c]);
        if (C.egAvg) {   // postStep's group time averages (radiation/RadiationIMC.hpp:1896-1902)
            const double norm = dt * A.vol[c];
            double *eg = C.egAvg + static_cast<size_t>(c) * C.groups;
            for (uint32_t g = 0; g < C.groups; ++g) eg[g] /= norm;
        }
        if (C.noFeedback) continue;
        double E = A.eint[c];
        if (E < 0.0) {   // throwIfNegativeInternalEnergy (:771-817)
            double thermalScale = C.arad * pow(A.T[c], 4.0) * A.vol[c];
            if (thermalScale < 1e-30) thermalScale = 1e-30;
            double ratio = fabs(E) / thermalScale;
            if (ratio < 0.1) {
                double fl = A.ceint[c];
                E = fl > 0.0 ? fl : 0.0;
                A.eint[c] = E;
            } else {
                raise_error(C, STORM_DERR_NEGATIVE_ENERGY, c, 0);
            }
        }
        // synchronizeMaterialCell (:830-866)
        const double spec = E / A.mass[c];
        A.ceint[c] = E;
        const double rho = A.mass[c] / A.vol[c];
        double T;
        if (M.eosKind == STORM_EOS_LINEAR) {
            T = (M.cvPerMass > 0.0) ? spec / M.cvPerMass : 0.0;
        } else {
            double ev = spec * rho;
            double rf = pow(rho, 1.0 - M.eosMu);
            double ratio = (ev > 0.0 ? ev : 0.0) / (M.eosF * rf);
            T = pow(ratio > 0.0 ? ratio : 0.0, 1.0 / M.eosBeta);
        }
        A.T[c] = T;
        if (C.withHydro) {   // cell.velocity = momentum / mass (:853-858)
            const double *m = C.mom + 3 * static_cast<size_t>(c);
            const double mass = A.mass[c];
            double4 v = C.vel[c];
            v.x = m[0] / mass;
            v.y = m[1] / mass;
            v.z = m[2] / mass;
            C.vel[c] = v;
        }
    }
}

// ------------------------------------------------------------------ replay
__global__ void k_replay(Ctx C, ReplayDev R, uint32_t n) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        Track T;
        PartReg &p = T.p;
        p.x = R.in[0][q]; p.y = R.in[1][q]; p.z = R.in[2][q];
        p.vx = R.in[3][q]; p.vy = R.in[4][q]; p.vz = R.in[5][q];
        p.t = R.in[6][q]; p.w = R.in[7][q]; p.w0 = R.in[8][q];
        p.cell = R.cell[q];
        p.nu = R.freq ? R.freq[q] : 0.0;
        track_begin(C, T);
        TapeRng rng{R.tape + R.tapeOffset[q], R.tapeLength[q], 0, false};
        LocalTally tal{0.0, 0.0, 0.0, 0.0, 0.0};
        PhysOut o = C.poly ? (C.withDDMC ? physics_step<5>(C, T, rng, tal) : physics_step<2>(C, T, rng, tal))
                           : (C.withHydro ? physics_step<3>(C, T, rng, tal) : physics_step<1>(C, T, rng, tal));
        R.phys[0][q] = p.x; R.phys[1][q] = p.y; R.phys[2][q] = p.z;
        R.phys[3][q] = p.vx; R.phys[4][q] = p.vy; R.phys[5][q] = p.vz;
        R.phys[6][q] = p.t; R.phys[7][q] = p.w;
        if (R.freqOut) R.freqOut[q] = p.nu;
        R.physStatus[q] = o.errCode ? -1 : o.status;
        R.physNext[q] = (o.status == CELL_MOVE && !o.errCode) ? (o.next != OUTSIDE ? o.next : o.ghost) : OUTSIDE;
        R.dep[0][q] = tal.mat_;
        R.dep[1][q] = tal.rad_;
        R.usedRW[q] = o.usedRW;
        R.draws[q] = rng.pos;
        if (R.momOut) {
            R.momOut[3 * static_cast<size_t>(q)] = tal.mx_;
            R.momOut[3 * static_cast<size_t>(q) + 1] = tal.my_;
            R.momOut[3 * static_cast<size_t>(q) + 2] = tal.mz_;
        }
        int m = o.errCode ? OUT_ERROR : (C.poly ? manager_handle<true>(C, T, o) : manager_handle<false>(C, T, o));
        R.mgr[0][q] = p.x; R.mgr[1][q] = p.y; R.mgr[2][q] = p.z;
        R.mgr[3][q] = p.vx; R.mgr[4][q] = p.vy; R.mgr[5][q] = p.vz;
        R.mgrCell[q] = p.cell;
        R.mgrStatus[q] = rng.exhausted() ? -2 : m;
    }
}

// ------------------------------------------------------------------ Random Walk tables
// RandomWalk::RandomWalk radius table (radiation/RandomWalk.hpp:41-78): one block
// per tau row; the 512-point radial CDF lives in shared memory.
__device__ double rw_radial_cdf(double x, double tau, double S) {   // computeRadialCDF :152-167
    if (tau <= 0.0) return (x > 0.0) ? 1.0 : 0.0;
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.0;
    if (tau < 0.01) {   // radialCdfFreeSpace :194-206
        double a = x / (2.0 * sqrt(tau));
        return clampd(erf(a) - 2.0 * a * exp(-a * a) / sqrt(RW_PI), 0.0, 1.0);
    }
    if (S < 1e-30) return 1.0;   // radialCdfEigen :208-237
    double sum = 0.0;
    for (int m = 1; m <= 500; ++m) {
        double arg = -static_cast<double>(m * m) * RW_PI * RW_PI * tau;
        if (arg < -700.0) break;
        double npi = static_cast<double>(m) * RW_PI;
        double npx = npi * x;
        double sn, cs;
        sincos(npx, &sn, &cs);
        sum += exp(arg) * (sn / npi - x * cs);
    }
    return clampd(2.0 * sum / S, 0.0, 1.0);
}
__global__ void k_rw_radius(const double *tau, const double *surv, double *radius) {
    __shared__ double g[RW_XGRID];
    const uint32_t row = blockIdx.x;
    const double t = tau[row];
    double S = t <= 0.0 || t < 1e-4 ? 1.0 : surv[row];
    // the eigen CDF normalises by computeSurvival(tau), which equals the table entry
    for (int k = threadIdx.x; k < RW_XGRID; k += blockDim.x)
        g[k] = rw_radial_cdf(static_cast<double>(k) / static_cast<double>(RW_XGRID - 1), t, S);
    __syncthreads();
    for (int j = threadIdx.x; j < RW_RADIUS; j += blockDim.x) {
        double xi = static_cast<double>(j) / static_cast<double>(RW_RADIUS - 1);
        double r;
        if (xi <= g[0]) r = 0.0;
        else if (xi >= g[RW_XGRID - 1]) r = 1.0;
        else {
            uint32_t first = 0, count = RW_XGRID;
            while (count > 0) {
                uint32_t step = count >> 1, it = first + step;
                if (g[it] < xi) { first = it + 1; count -= step + 1; } else count = step;
            }
            if (first == 0) first = 1;
            double g0 = g[first - 1], g1 = g[first];
            double x0 = static_cast<double>(first - 1) / static_cast<double>(RW_XGRID - 1);
            double x1 = static_cast<double>(first) / static_cast<double>(RW_XGRID - 1);
            double f = (g1 > g0) ? (xi - g0) / (g1 - g0) : 0.5;
            r = x0 + f * (x1 - x0);
        }
        radius[static_cast<size_t>(row) * RW_RADIUS + j] = r;
    }
}
__global__ void k_rw_sample(RwTables T, uint32_t n, const double *xiLeak, const double *tau, const double *xiRad,
                            double *leak, double *rad) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        if (xiLeak) leak[q] = rw_sample_leak(T, xiLeak[q]);
        if (tau && xiRad) rad[q] = rw_sample_radius(T, tau[q], xiRad[q]);
    }
}

// ------------------------------------------------------------------ launchers
static inline uint32_t grid_for(uint64_t n, uint32_t block, uint32_t cap) {
    uint64_t g = (n + block - 1) / block;
    if (g == 0) g = 1;
    return static_cast<uint32_t>(g < cap ? g : cap);
}

void launch_begin(cudaStream_t s, const Bank &b, uint32_t n, uint32_t pidOffset, double dt, DevStats *st,
                  uint32_t lo) {
    if (n > lo) k_begin<<<grid_for(n - lo, 256, 4096), 256, 0, s>>>(b, lo, n, pidOffset, dt, st);
}
void launch_prestep(cudaStream_t s, const Ctx &C, const CellArrays &A, const OpacityEos &M, double dt) {
    k_prestep<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A, M, dt);
}
void launch_ddmc_rates(cudaStream_t s, const Ctx &C, const CellArrays &A) {
    k_ddmc_rates<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A);
}
void launch_rw_eligibility(cudaStream_t s, const Ctx &C, const CellArrays &A) {
    k_rw_eligibility<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A);
}
void launch_emission_energy(cudaStream_t s, const Ctx &C, const CellArrays &A, double dt) {
    k_emission_energy<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A, dt);
}
void launch_sequential_sum(cudaStream_t s, const double *v, uint32_t n, double *out) {
    k_sequential_sum<<<1, 256, 0, s>>>(v, n, out, nullptr);
}
void launch_sequential_sum_if(cudaStream_t s, const double *v, uint32_t n, double *out, const int32_t *onlyIf) {
    k_sequential_sum<<<1, 256, 0, s>>>(v, n, out, onlyIf);
}
void launch_allocate_checked(cudaStream_t s, const Ctx &C, const CellArrays &A, const double *total,
                             uint64_t newPerCell, double rel, int32_t *ambiguous) {
    k_allocate_checked<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A, total, newPerCell, rel, ambiguous);
}
void launch_allocate(cudaStream_t s, const Ctx &C, const CellArrays &A, const double *total, uint64_t newPerCell) {
    k_allocate<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A, total, newPerCell, nullptr);
}
void launch_allocate_if(cudaStream_t s, const Ctx &C, const CellArrays &A, const double *total, uint64_t newPerCell,
                        const int32_t *onlyIf) {
    k_allocate<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A, total, newPerCell, onlyIf);
}
void launch_emission_debit(cudaStream_t s, const Ctx &C, const CellArrays &A, DevStats *st) {
    k_emission_debit<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A, st);
}
void launch_scan_u64(cudaStream_t s, const uint64_t *in, uint32_t n, uint64_t *out, uint64_t *tileSums, uint64_t *total) {
    const uint32_t tiles = (n + 1023) / 1024 ? (n + 1023) / 1024 : 1;
    k_scan_tiles<<<tiles, 1024, 0, s>>>(in, n, out, tileSums);
    k_scan_sums<<<1, 1024, 0, s>>>(tileSums, tiles, total);
    k_scan_add<<<tiles, 1024, 0, s>>>(out, n, tileSums, total);
}
void launch_emit_cells(cudaStream_t s, const Ctx &C, const CellArrays &A, const uint64_t *offsets, uint64_t eBegin,
                       uint64_t count, const Bank &b, uint32_t bankBase, uint32_t pidBase, double dt, DevStats *st) {
    if (!count) return;
    if (C.fp32 && !C.poly)   // polyhedral cells: the FP64 sampler, then the cell frame
        k_emit_cells32<<<grid_for(count, 256, 148 * 16), 256, 0, s>>>(C, A, offsets, eBegin, count, b, bankBase,
                                                                      pidBase, dt, st);
    else
        k_emit_cells<<<grid_for(count, 256, 148 * 16), 256, 0, s>>>(C, A, offsets, eBegin, count, b, bankBase, pidBase,
                                                                    dt, st);
}
__global__ void k_set_u32(uint32_t *p, uint32_t v) { *p = v; }
void launch_set_u32(cudaStream_t s, uint32_t *p, uint32_t v) { k_set_u32<<<1, 1, 0, s>>>(p, v); }
void launch_poly_tets(cudaStream_t s, const Ctx &C, const uint32_t *tetOff, double *tetCum, uint2 *tetAT) {
    k_poly_tets<<<grid_for(C.ncells, 128, 8192), 128, 0, s>>>(C, tetOff, tetCum, tetAT);
}
void launch_emit_faces(cudaStream_t s, const Ctx &C, const FaceSources &F, uint64_t fBegin, uint64_t count,
                       const Bank &b, uint32_t bankBase, uint32_t pidBase, double dt, DevStats *st) {
    if (!count) return;
    k_emit_faces<<<grid_for(count, 256, 148 * 16), 256, 0, s>>>(C, F, fBegin, count, b, bankBase, pidBase, dt, st);
}
void launch_face_spectra(cudaStream_t s, const Ctx &C, double *cdf) { k_face_spectra<<<1, 32, 0, s>>>(C, cdf); }
void launch_strat_keys(cudaStream_t s, const Ctx &C, const CensusBank &cen, uint32_t n, uint64_t *keys, uint32_t *vals,
                       uint32_t combKey, int pidBits, const StratParams &S, double *wc) {
    k_strat_keys<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(C, cen, n, keys, vals, combKey, pidBits, S, wc);
}
void launch_strat_sums(cudaStream_t s, const double *wS, const uint32_t *start, uint32_t ncells, uint32_t bins,
                       double *binW, double *cellW) {
    k_strat_sums<<<grid_for(ncells, 256, 8192), 256, 0, s>>>(wS, start, ncells, bins, binW, cellW);
}
void launch_strat_plan(cudaStream_t s, const Ctx &C, const CombParams &P, const StratParams &S, const double *wS,
                       const uint32_t *start, const double *binW, const double *cellW, const double *Wtot,
                       uint32_t *pCount, double *pWeight, uint64_t *cellCount, double *eradCensus, DevStats *st) {
    k_strat_plan<<<grid_for(C.ncells, 128, 8192), 128, 0, s>>>(C, P, S, wS, start, binW, cellW, Wtot, pCount, pWeight,
                                                             cellCount, eradCensus, st);
}
void launch_transport(cudaStream_t s, uint32_t grid, const Ctx &C, const Bank &in, const uint32_t *nIn, const Bank &out,
                      uint32_t *nOut, const CensusBank &cen, uint32_t *nCen, uint32_t K, DevStats *st, int minBlocks) {
    if (C.fp32) {
        switch (minBlocks) {
        case 3: k_transport32<3><<<grid, 256, 0, s>>>(C, in, nIn, out, nOut, cen, nCen, K, st); break;
        case 4: k_transport32<4><<<grid, 256, 0, s>>>(C, in, nIn, out, nOut, cen, nCen, K, st); break;
        case 2: k_transport32<2><<<grid, 256, 0, s>>>(C, in, nIn, out, nOut, cen, nCen, K, st); break;
        default: k_transport32<1><<<grid, 256, 0, s>>>(C, in, nIn, out, nOut, cen, nCen, K, st); break;
        }
        return;
    }
    switch (minBlocks) {
    case 3: k_transport<3><<<grid, 256, 0, s>>>(C, in, nIn, out, nOut, cen, nCen, K, st); break;
    case 4: k_transport<4><<<grid, 256, 0, s>>>(C, in, nIn, out, nOut, cen, nCen, K, st); break;
    case 2: k_transport<2><<<grid, 256, 0, s>>>(C, in, nIn, out, nOut, cen, nCen, K, st); break;
    default: k_transport<1><<<grid, 256, 0, s>>>(C, in, nIn, out, nOut, cen, nCen, K, st); break;
    }
}
int transport_blocks_per_sm(int minBlocks, bool fp32) {
    int nb = 0;
    if (fp32) {
        switch (minBlocks) {
        case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport32<3>, 256, 0); break;
        case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport32<4>, 256, 0); break;
        case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport32<2>, 256, 0); break;
        default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport32<1>, 256, 0); break;
        }
        return nb;
    }
    switch (minBlocks) {
    case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport<3>, 256, 0); break;
    case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport<4>, 256, 0); break;
    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport<2>, 256, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport<1>, 256, 0); break;
    }
    return nb;
}
void launch_comb_keys(cudaStream_t s, const Ctx &C, const CensusBank &cen, uint32_t n, uint64_t *keys, uint32_t *vals,
                      uint32_t combKey, int pidBits, double *wc) {
    k_comb_keys<<<grid_for(n, 256, 8192), 256, 0, s>>>(C, cen, n, keys, vals, combKey, pidBits, wc);
}
int launch_radix_sort(cudaStream_t s, uint64_t *keys, uint32_t *vals, uint64_t *keysAlt, uint32_t *valsAlt, uint32_t n,
                      int bits, uint32_t *tileHist) {
    // returns 1 when the sorted data ends in the Alt buffers
    // the scatter stages a tile in more than the default 48 KB of shared memory (set on the current device)
    cudaFuncSetAttribute(k_rs_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(RS_SMEM));
    const uint32_t ntiles = (n + RS_TILE - 1) / RS_TILE ? (n + RS_TILE - 1) / RS_TILE : 1;
    int passes = (bits + 7) / 8;
    uint64_t *ka = keys, *kb = keysAlt;
    uint32_t *va = vals, *vb = valsAlt;
    const uint32_t len = 256 * ntiles;
    const uint32_t stiles = (len + 1023) / 1024;
    uint64_t *scanSums = reinterpret_cast<uint64_t *>(tileHist + len + (len & 1));
    for (int p = 0; p < passes; ++p) {
        k_rs_hist<<<ntiles, RS_THREADS, 0, s>>>(ka, n, 8 * p, tileHist, ntiles);
        k_scan32_tiles<<<stiles, 1024, 0, s>>>(tileHist, len, scanSums);
        k_scan_sums<<<1, 1024, 0, s>>>(scanSums, stiles, scanSums + stiles);
        k_scan32_add<<<stiles, 1024, 0, s>>>(tileHist, len, scanSums);
        k_rs_scatter<<<ntiles, RS_THREADS, RS_SMEM, s>>>(ka, va, kb, vb, n, 8 * p, tileHist, ntiles);
        uint64_t *tk = ka; ka = kb; kb = tk;
        uint32_t *tv = va; va = vb; vb = tv;
    }
    return passes & 1;
}
// Bucket sort of the comb keys (see k_bucket_count).  `start` receives the
// first position of every run 0..nRuns (start[nRuns]: the first key outside
// every run); `cursor` is scratch of nRuns + 1 words and `scanSums` of
// bucket_scan_words(nRuns + 1).  The sorted pairs end in (outKeys, outVals)
// and the census weights in sorted order in wS (positions below start[nRuns]).
// Long runs are listed in longRuns (longCap entries); flags[0] counts them and
// flags[1] is set when a run is too long for this sort (then nothing is sorted
// and the caller falls back to launch_radix_sort).
void launch_bucket_sort(cudaStream_t s, const Ctx &C, const CensusBank &cen, const uint64_t *keys, uint32_t n,
                        int pidBits, uint32_t nRuns, uint32_t *start, uint32_t *cursor, uint64_t *scanSums,
                        uint64_t *outKeys, uint32_t *outVals, double *wS, uint32_t *longRuns, uint32_t longCap,
                        uint32_t *flags, const double *wc) {
    const uint32_t len = nRuns + 1;
    cudaMemsetAsync(start, 0, sizeof(uint32_t) * len, s);
    cudaMemsetAsync(flags, 0, 2 * sizeof(uint32_t), s);
    k_bucket_count<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(keys, n, pidBits, nRuns, start);
    const uint32_t stiles = (len + 1023) / 1024;
    k_scan32_tiles<<<stiles, 1024, 0, s>>>(start, len, scanSums);
    k_scan_sums<<<1, 1024, 0, s>>>(scanSums, stiles, scanSums + stiles);
    k_scan32_add<<<stiles, 1024, 0, s>>>(start, len, scanSums);
    cudaMemcpyAsync(cursor, start, sizeof(uint32_t) * len, cudaMemcpyDeviceToDevice, s);
    k_bucket_place<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(keys, n, pidBits, nRuns, cursor, outKeys, outVals);
    k_bucket_sort_runs<<<grid_for(nRuns, BUCKET_WARPS, 148 * 32), 32 * BUCKET_WARPS, 0, s>>>(
        C, cen, wc, outKeys, outVals, wS, start, nRuns, pidBits, longRuns, flags, longCap);
    const size_t smem = sizeof(uint64_t) * BUCKET_BLOCK_MAX;
    cudaFuncSetAttribute(k_bucket_sort_long, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    k_bucket_sort_long<<<148, 256, smem, s>>>(C, cen, wc, outKeys, outVals, wS, start, pidBits, longRuns, flags,
                                              longCap, flags + 1);
}
size_t bucket_scan_words(uint32_t len) { return (len + 1023) / 1024 + 2; }
uint32_t bucket_long_capacity(uint32_t n) { return n / (BUCKET_WARP_MAX + 1) + 1; }

uint32_t radix_tile_count(uint32_t n) { return (n + RS_TILE - 1) / RS_TILE ? (n + RS_TILE - 1) / RS_TILE : 1; }
// 32-bit words the radix sort needs for its tile histogram and the scan's tile sums
size_t radix_scratch_words(uint32_t n) {
    size_t len = 256ull * radix_tile_count(n);
    size_t stiles = (len + 1023) / 1024;
    return len + (len & 1) + 2 * (stiles + 2);
}
void launch_comb_ranges(cudaStream_t s, const uint64_t *keys, uint32_t n, uint32_t ncells, uint32_t *start, int pidBits) {
    k_comb_ranges<<<grid_for(ncells + 1, 256, 8192), 256, 0, s>>>(keys, n, ncells, start, pidBits);
}
void launch_sorted_weights(cudaStream_t s, const Ctx &C, const CensusBank &cen, const uint32_t *idx, uint32_t n,
                           double *wS) {
    if (n) k_sorted_weights<<<grid_for(n, 256, 8192), 256, 0, s>>>(C, cen, idx, n, wS);
}
void launch_comb_cell_sums(cudaStream_t s, const double *wS, const uint32_t *start, uint32_t ncells, double *W) {
    k_comb_cell_sums<<<grid_for(ncells, 128, 8192), 128, 0, s>>>(wS, start, ncells, W);
}
void launch_blocked_sum(cudaStream_t s, const double *v, uint32_t n, double *out) {
    k_blocked_sum<<<1, 1024, 0, s>>>(v, n, out);
}
void launch_comb_plan(cudaStream_t s, const Ctx &C, const CombParams &P, const double *wS, const uint32_t *start,
                      const double *W, const double *Wtot, uint32_t *pCount, double *pWeight, uint64_t *cellCount,
                      double *eradCensus, DevStats *st) {
    k_comb_plan<<<grid_for(C.ncells, 128, 8192), 128, 0, s>>>(C, P, wS, start, W, Wtot, pCount, pWeight, cellCount,
                                                               eradCensus, st);
}
void launch_comb_emit(cudaStream_t s, const Ctx &C, const CensusBank &cen, const uint32_t *idx, const uint64_t *sortedKeys,
                      int pidBits, uint32_t bins, uint32_t nValid, const uint32_t *pCount, const double *pWeight,
                      const uint64_t *pOffset, const Bank &out) {
    if (!nValid) return;
    if (C.fp32)
        k_comb_emit<true><<<grid_for(nValid, 256, 148 * 16), 256, 0, s>>>(C, cen, idx, sortedKeys, pidBits, bins, nValid, pCount,
                                                                           pWeight, pOffset, out);
    else
        k_comb_emit<false><<<grid_for(nValid, 256, 148 * 16), 256, 0, s>>>(C, cen, idx, sortedKeys, pidBits, bins, nValid, pCount,
                                                                            pWeight, pOffset, out);
}
// The same write, output-driven (k_comb_emit_out).  src: scratch of `total`
// words; tileMax: scratch of total / 1024 + 1 words.
void launch_comb_emit_out(cudaStream_t s, const Ctx &C, const CensusBank &cen, const uint32_t *idx,
                          const uint64_t *sortedKeys, int pidBits, uint32_t bins, uint32_t nValid, uint32_t total,
                          const uint32_t *pCount, const double *pWeight, const uint64_t *pOffset, uint32_t *src,
                          uint32_t *tileMax, const Bank &out) {
    if (!nValid || !total) return;
    cudaMemsetAsync(src, 0, sizeof(uint32_t) * total, s);
    k_emit_src_mark<<<grid_for(nValid, 256, 148 * 16), 256, 0, s>>>(pCount, pOffset, nValid, src);
    const uint32_t tiles = (total + 1023) / 1024;
    k_max_tiles<<<tiles, 1024, 0, s>>>(src, total, tileMax);
    k_max_tile_prefix<<<1, 1024, 0, s>>>(tileMax, tiles);
    k_max_apply<<<tiles, 1024, 0, s>>>(src, total, tileMax);
    if (C.fp32)
        k_comb_emit_out<true><<<grid_for(total, 256, 148 * 16), 256, 0, s>>>(C, cen, idx, sortedKeys, pidBits, bins, total,
                                                                             src, pCount, pWeight, out);
    else
        k_comb_emit_out<false><<<grid_for(total, 256, 148 * 16), 256, 0, s>>>(C, cen, idx, sortedKeys, pidBits, bins,
                                                                              total, src, pCount, pWeight, out);
}
void launch_mask_count_upto(cudaStream_t s, const uint32_t *pCount, uint32_t n, const uint32_t *nValid, uint64_t *out) {
    k_mask_count_upto<<<grid_for(n, 256, 8192), 256, 0, s>>>(pCount, n, nValid, out);
}
void launch_census_keys_pid(cudaStream_t s, const Ctx &C, const CensusBank &cen, uint32_t n, uint64_t *keys,
                            uint32_t *vals) {
    k_census_keys_pid<<<grid_for(n, 256, 8192), 256, 0, s>>>(C, cen, n, keys, vals);
}
void launch_gather(cudaStream_t s, const Ctx &C, const CensusBank &src, const uint32_t *idx, uint32_t n, const Bank &dst,
                   double *eradCensus, DevStats *st) {
    k_gather<<<grid_for(n, 256, 8192), 256, 0, s>>>(C, src, idx, n, dst, eradCensus, st);
}
template <class F>
static void refill_launch(cudaStream_t s, uint32_t grid, int minBlocks, const Ctx &C, const Bank &in, uint32_t n,
                          uint32_t *nextIdx, const CensusBank &cen, uint32_t *nCen, uint32_t burst, uint32_t maxSegs,
                          DevStats *st) {
    switch (minBlocks) {
    case 4: k_transport_refill<F, 4><<<grid, 256, 0, s>>>(C, in, n, nextIdx, cen, nCen, burst, maxSegs, st); break;
    case 3: k_transport_refill<F, 3><<<grid, 256, 0, s>>>(C, in, n, nextIdx, cen, nCen, burst, maxSegs, st); break;
    case 2: k_transport_refill<F, 2><<<grid, 256, 0, s>>>(C, in, n, nextIdx, cen, nCen, burst, maxSegs, st); break;
    default: k_transport_refill<F, 1><<<grid, 256, 0, s>>>(C, in, n, nextIdx, cen, nCen, burst, maxSegs, st); break;
    }
}
void launch_transport_refill(cudaStream_t s, uint32_t grid, int minBlocks, const Ctx &C, const Bank &in, uint32_t n,
                             uint32_t *nextIdx, const CensusBank &cen, uint32_t *nCen, uint32_t burst, uint32_t maxSegs,
                             DevStats *st) {
    if (C.egAvg) {   // multigroup problems with the group time averages
        if (C.fp32 && C.withDDMC) refill_launch<Form32MGEg>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.fp32) refill_launch<Form32MGLeanEg>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.withHydro) refill_launch<Form64HydroEg>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.withDDMC) refill_launch<Form64FullEg>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else refill_launch<Form64MGEg>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        return;
    }
    if (C.fixMat) {   // reproducible tallies
        if (C.fp32 && C.poly && C.withDDMC) refill_launch<Form32PolyDDMCFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.fp32 && C.poly) refill_launch<Form32PolyFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.fp32 && C.groups >= 2 && C.withDDMC) refill_launch<Form32MGFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.fp32 && C.groups >= 2) refill_launch<Form32MGLeanFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.fp32 && C.withDDMC) refill_launch<Form32Fix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.fp32) refill_launch<Form32LeanFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.poly && C.withDDMC) refill_launch<Form64PolyDDMCFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.poly) refill_launch<Form64PolyFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.groups >= 2 && !C.withDDMC) refill_launch<Form64MGFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else if (C.groups >= 2 || C.withDDMC) refill_launch<Form64FullFix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        else refill_launch<Form64Fix>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
        return;
    }
    if (C.fp32 && C.poly && C.withDDMC) refill_launch<Form32PolyDDMC>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.fp32 && C.poly) refill_launch<Form32Poly>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.fp32 && C.groups >= 2 && C.withDDMC) refill_launch<Form32MG>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.fp32 && C.groups >= 2) refill_launch<Form32MGLean>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.fp32 && C.withDDMC) refill_launch<Form32>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.fp32) refill_launch<Form32Lean>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.poly && C.withDDMC) refill_launch<Form64PolyDDMC>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.poly) refill_launch<Form64Poly>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.withHydro) refill_launch<Form64Hydro>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.groups >= 2 && !C.withDDMC) refill_launch<Form64MG>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else if (C.groups >= 2 || C.withDDMC) refill_launch<Form64Full>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
    else refill_launch<Form64>(s, grid, minBlocks, C, in, n, nextIdx, cen, nCen, burst, maxSegs, st);
}
template <class F>
static int refill_occ(int minBlocks) {
    int nb = 0;
    switch (minBlocks) {
    case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport_refill<F, 4>, 256, 0); break;
    case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport_refill<F, 3>, 256, 0); break;
    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport_refill<F, 2>, 256, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_transport_refill<F, 1>, 256, 0); break;
    }
    return nb;
}
int refill_blocks_per_sm(int minBlocks, bool fp32) { return fp32 ? refill_occ<Form32>(minBlocks) : refill_occ<Form64>(minBlocks); }

// Count (per warp) the census entries whose cell index is not a cell of the grid.
__global__ void k_count_bad_cells(const uint32_t *cell, uint32_t n, uint32_t N, int32_t *bad) {
    bool b = false;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) b |= cell[q] >= N;
    if (__any_sync(FULL, b) && (threadIdx.x & 31) == 0) atomicAdd(bad, 1);
}
__global__ void k_to_float(const double *src, float *dst, uint32_t n) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        dst[q] = static_cast<float>(src[q]);
}
void launch_to_float(cudaStream_t s, const double *src, float *dst, uint32_t n) {
    if (n) k_to_float<<<grid_for(n, 256, 4096), 256, 0, s>>>(src, dst, n);
}
// Particles per cell at the start of transport (MonteCarloManagerSerial's
// beginningParticleCount_, manager/MonteCarloManagerSerial.hpp:419-424).
__global__ void k_cell_histogram(const uint32_t *cell, uint32_t n, uint32_t N, uint32_t *count) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t c = cell[q];
        if (c < N) atomicAdd(count + c, 1u);
    }
}
void launch_cell_histogram(cudaStream_t s, const uint32_t *cell, uint32_t n, uint32_t N, uint32_t *count) {
    if (n) k_cell_histogram<<<grid_for(n, 256, 8192), 256, 0, s>>>(cell, n, N, count);
}
void launch_shard_pack_runs(cudaStream_t s, const double *runW, const uint32_t *start, uint32_t nRuns, double *x) {
    k_shard_pack_runs<<<grid_for(nRuns, 256, 8192), 256, 0, s>>>(runW, start, nRuns, x);
}
void launch_shard_cell_weights(cudaStream_t s, const double *x, uint32_t ncells, uint32_t shards, double *Wc) {
    k_shard_cell_weights<<<grid_for(ncells, 256, 8192), 256, 0, s>>>(x, ncells, shards, Wc);
}
void launch_comb_plan_sharded(cudaStream_t s, const Ctx &C, const CombParams &P, const double *wS,
                              const uint32_t *start, const double *x, const double *Wc, const double *Wtot,
                              uint32_t lo, uint32_t hi, uint32_t *pCount, double *pWeight, double *eradCensus,
                              DevStats *st) {
    k_comb_plan_sharded<<<grid_for(C.ncells, 128, 8192), 128, 0, s>>>(C, P, wS, start, x, Wc, Wtot, lo, hi, pCount,
                                                                      pWeight, eradCensus, st);
}
void launch_shard_pack_census(cudaStream_t s, const uint64_t *pOff, const uint64_t *total, const uint32_t *start,
                              uint32_t n, uint32_t ncells, uint32_t shards, uint32_t lo, uint32_t hi,
                              const double *eradCensus, double *x) {
    const uint32_t m = ncells > shards ? ncells : shards;
    k_shard_pack_census<<<grid_for(m, 256, 8192), 256, 0, s>>>(pOff, total, start, n, ncells, shards, lo, hi,
                                                                eradCensus, x);
}
void launch_add_into(cudaStream_t s, double *y, const double *x, uint32_t n) {
    if (n) k_add_into<<<grid_for(n, 256, 8192), 256, 0, s>>>(y, x, n);
}
void launch_count_bad_cells(cudaStream_t s, const uint32_t *cell, uint32_t n, uint32_t N, int32_t *bad) {
    if (n) k_count_bad_cells<<<grid_for(n, 256, 4096), 256, 0, s>>>(cell, n, N, bad);
}
void launch_bank_to_local(cudaStream_t s, const Ctx &C, const Bank &src, const Bank &dst, uint32_t n, uint32_t lo) {
    if (n > lo) k_bank_to_local<<<grid_for(n - lo, 256, 8192), 256, 0, s>>>(C, src, dst, lo, n);
}
void launch_bank_to_census(cudaStream_t s, const Ctx &C, const Bank &src, const CensusBank &dst, uint32_t n) {
    if (n) k_bank_to_census<<<grid_for(n, 256, 8192), 256, 0, s>>>(C, src, dst, n);
}
void launch_bank_to_global(cudaStream_t s, const Ctx &C, const Bank &src, const Bank &dst, uint32_t n) {
    if (n) k_bank_to_global<<<grid_for(n, 256, 8192), 256, 0, s>>>(C, src, dst, n);
}
void launch_poststep(cudaStream_t s, const Ctx &C, const CellArrays &A, const OpacityEos &M, double dt) {
    k_poststep<<<grid_for(C.ncells, 256, 8192), 256, 0, s>>>(C, A, M, dt);
}
void launch_replay(cudaStream_t s, const Ctx &C, const ReplayDev &R, uint32_t n) {
    k_replay<<<grid_for(n, 128, 8192), 128, 0, s>>>(C, R, n);
}
void launch_rw_radius(cudaStream_t s, const double *tau, const double *surv, double *radius) {
    k_rw_radius<<<RW_TABLE, 256, 0, s>>>(tau, surv, radius);
}
void launch_rw_sample(cudaStream_t s, const RwTables &T, uint32_t n, const double *xiLeak, const double *tau,
                      const double *xiRad, double *leak, double *rad) {
    k_rw_sample<<<grid_for(n, 256, 4096), 256, 0, s>>>(T, n, xiLeak, tau, xiRad, leak, rad);
}

}  // namespace storm
