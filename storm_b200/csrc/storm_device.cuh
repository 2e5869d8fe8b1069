// Device-side building blocks of the IMC engine: counter-based random streams,
// the per-cell / mesh context, and the FP64 segment (one RadiationIMC::step call
// plus the serial manager's face and boundary handling).
//
// This translation unit is compiled with --fmad=false: every plain expression
// rounds like the reference's x86-64 build (no contraction), and expressions keep
// the reference's association, so on the same uniforms a segment reproduces the
// reference bit for bit except where CUDA's log1p / expm1 / sin / cos / exp / log
// differ from glibc by an ulp.
#pragma once

#include <cstdint>
#include <cfloat>
#include <math_constants.h>

#include "storm_cuda.h"

namespace storm {

// ParticleStatus (particle/ParticleStatus.hpp:8-15)
enum : int { NO_CELL_MOVE = 0, CELL_MOVE = 1, DONE = 2, REMOVE = 3, REFLECT = 4 };
// outcome of a segment after the manager's handling
enum : int { OUT_CONTINUE = 0, OUT_CENSUS = 1, OUT_CUTOFF = 2, OUT_ESCAPE = 3, OUT_ERROR = -1 };
// random stream tags
enum : uint32_t { TAG_TRANSPORT = 1, TAG_CELL_EMIT = 2, TAG_FACE_EMIT = 3, TAG_COMB = 4 };

constexpr uint32_t OUTSIDE = 0xffffffffu;
constexpr double EPSILON_FACE = 1e-12;       // particle/Particle.hpp:17
constexpr double MONTECARLO_EPS = 1e-8;      // manager/MonteCarloConfig.hpp:11
constexpr double RW_NUDGE = 1e-6;            // radiation/RadiationIMC.hpp:1211
constexpr float ENTRY32 = 1.0f - 0x1p-21f;    // FP32 form: entry offset / half width after a cell change
constexpr double RW_PI = 3.14159265358979323846;
constexpr double TWO_PI_ISO = 6.283185307179586476925286766559;   // radiation/RadiationOpacityModel.hpp:143
constexpr double ONE_BELOW = 0x1.fffffffffffffp-1;                  // std::nextafter(1.0, 0.0)
constexpr int RW_TABLE = 1024;
constexpr int RW_RADIUS = 256;
constexpr int RW_XGRID = 512;
constexpr int RW_SHRINK_CAP = 100000;

// One box face as the host precomputes it from BoundaryCondition's helpers
// (boundary/BoundaryCondition.hpp:61-108) with the reference's arithmetic.
struct BoxFaceDev {
    double raw[3];      // CrossProduct(v1 - v0, v2 - v0)
    double unit[3];     // raw * (1 / |raw|), oriented toward the box centre
    double on[3];       // vertices[0]
    double thresh;      // EPSILON * faceScale^3
    double nudge;       // 1e-6 * faceScale
    int32_t action;     // StormFaceAction
    int32_t valid;      // the helper's finiteness / non-degeneracy checks
};

// The leak-time samplers look for the first table entry whose survival is at
// most 1 - xi.  A bucket table over the survival value gives, for each of
// RW_LEAK_BUCKETS equal intervals of it, the number of entries above the
// interval's top, where a short walk forward to the answer starts: the same
// entry a binary search finds, in about one step instead of ten dependent loads.
constexpr int RW_LEAK_BUCKETS = 4096;
struct RwTables {
    const double *tau, *logTau, *surv, *radius;
    double logMin, logMax;   // std::log(1e-8), std::log(64) as the host computes them
    // FP32 copies for the FP32-tracking form
    const float *logTau32, *surv32, *radius32;
    const uint16_t *leakStart, *leakStart32;   // per bucket: entries of surv (surv32) above its top
};

// Everything a kernel needs, passed by value.
struct Ctx {
    uint32_t nx, ny, nz, ncells;
    const double *xe, *ye, *ze, *xc, *yc, *zc;
    double X0, X1, Y0, Y1, Z0, Z1;
    BoxFaceDev bf[6];
    int32_t escapeNoCheck;
    int32_t withRW;
    int32_t noFeedback;
    int32_t perCellCounters;
    // moving material (withHydro): per cell (vx, vy, vz, gamma) and the cells' momentum (3 per cell)
    int32_t withHydro;
    double4 *vel;
    double *mom;
    double invC2;                  // units::inv_clight2
    // particle shards (storm_cuda_set_sharding): 1 = the whole problem on this handle
    uint32_t shards;
    const uint64_t *shardBounds;   // 3 (shards + 1) pid bounds: census, cell packets, face packets
    double clight, arad, sigmaSB, kevKelvin;
    double rwMinParticle, rwMinCell;
    double sourceT[6];       // source temperature of each box face [K]
    uint32_t seedLo, seedHi, step;
    // FP32-tracking form
    int32_t fp32;            // banks hold cell-local FP32 offsets and FP32 directions
    const float *hx, *hy, *hz;   // half widths per axis
    const float4 *phys32;    // x = 1/sigma_e (inf when none), y = sigma_a f [1/cm], z = RW reach, w = -1/(sigma_a f c)
    float rwDiffPerReach;    // c / (3 rwMinParticleOpticalDepth): diffusion coefficient = reach * this
    float reflNudge[6];      // 1e-6 * faceScale of each box face, capped at a quarter cell
    double invC;             // 1 / c
    // per-cell arrays
    const double4 *phys;     // per-cell segment constants (CellPhys layout)
    const double *sigA, *sigS, *fleck, *rwSigT;
    const uint8_t *rwElig;
    double *eint, *eradAvg;
    uint32_t *segs;
    RwTables rw;
    int32_t *err;            // [0] code, [1] cell lo, [2] particle lo
    // multigroup (groups >= 2)
    uint32_t groups;
    int32_t mgGroupConst;    // opacity at the centre of the particle's group
    const double *gb;        // groups + 1 bounds [erg]
    double mgP, mgQ, mgS, kBoltz;
    const double *T;         // cell temperatures
    const double *sig0;      // sigma0 per cell
    const double *mgCdf;     // per cell, groups + 1: cumulative sigma_g B_g (the emission spectrum)
    const double4 *pgrw;     // per cell: sigmaT_bar, sigmaA_bar, D, gamma
    const uint32_t *pgrwCut; // per cell: group cutoff (0 = no PGRW)
    const float *gb32;       // FP32-tracking form: bounds and group centres as floats
    const float *gc32;
    const double *faceCdf;   // per box face, groups + 1: cumulative B_g at the face's source temperature
    const double *mgEp;      // per group: E_g^p at the group centre (host pow, the opacity model's value)
    const float *mgEp32;     // the same as floats, FP32-tracking form
    double *egAvg;           // group time averages (withEgTimeAvg): ncells x groups, NULL when off
    // reproducible tallies: 4 fixed-point limbs per cell for the deposits and for
    // Erad_time_avg (NULL when off), and this step's power-of-two scales into them
    unsigned long long *fixMat, *fixRad;
    double fixScaleMat, fixScaleRad;
    double *mgKTq;           // per cell: (kT)^q, written by the prestep
    // DDMC-style leakage (RadiationIMCParameters::withDDMC)
    int32_t withDDMC;
    int32_t ddmcPgrw;        // ddmcUseMultigroupPGRW with a multigroup opacity
    double ddmcMinParticle, ddmcMinCell;
    double4 *ddmc;           // per cell: sigma_T, sigma_A, eligible (1/0), D  (prestep)
    double *ddmcTot;         // per cell: total leak rate [1/s], 0 where not eligible
    double *ddmcRate;        // per cell x 6 faces in GetCellFaces order (polyhedral: per cell-face slot):
                             // leak rate, 0 where none
    float *ddmcCum32;        // FP32 form on a polyhedral mesh, per cell-face slot: cumulative leak fraction
    const double *cfA;       // polyhedral mesh, per cell-face slot: the face's area (GetArea)
    uint32_t *ddmcCut;       // per cell: group cutoff (multigroup PGRW form)
    float4 *ddmc32;          // FP32 form, 3 per cell: (reach, 1/total, sigma_A f c, frequency bound),
                             // (cumulative face fractions 0-3), (fractions 4-5, last leak face, 0)
    // convex-polyhedral mesh (poly != 0; nx = ncells, ny = nz = 1 so cell_ijk stays in range)
    int32_t poly;
    const uint32_t *cfo;     // per cell: its first cell-face slot (ncells + 1)
    const double4 *cfN;      // per cell-face slot: the inward unit normal of updateGridData
    const double4 *cfP;      // per cell-face slot: the face centroid (FaceCM)
    const uint32_t *cfNext;  // per cell-face slot: the neighbour cell, or a ghost >= ncells
    const uint32_t *cfFace;  // per cell-face slot: the global face index
    const double *mpx, *mpy, *mpz;   // mesh points (GetMeshPoint)
    const uint32_t *fvo, *fvi;       // face polygons: offsets (nfaces + 1) and vertex indices
    const double *vtx;       // polygon vertices, 3 per vertex
    const double *chord;     // per cell: 4 V / S
    const float4 *cfN32;     // FP32 form, per cell-face slot: inward unit normal and the distance of the
                             // cell's mesh point from the face plane, (mesh point - faceCM).n
    // polyhedral cell emission: each cell's fan tetrahedra in the sampler's order
    // (faces in GetCellFaces order, triangles (v0, v_t, v_t+1)) with their running
    // volume sums, and each tetrahedron's (first, t) offsets into fvi
    const uint32_t *tetOff;  // per cell: its first tetrahedron (ncells + 1)
    const double *tetCum;
    const uint2 *tetAT;
};

// ------------------------------------------------------------------ errors
__device__ __forceinline__ void raise_error(const Ctx &C, int code, uint32_t cell, uint32_t particle) {
    if (atomicCAS(C.err, 0, code) == 0) {
        C.err[1] = static_cast<int32_t>(cell);
        C.err[2] = static_cast<int32_t>(particle);
    }
}

// ------------------------------------------------------------------ Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                              uint32_t k1, uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        // one 32x32->64 multiply gives both halves of each product
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// 52-bit uniform on the open interval: (m + 0.5) * 2^-52.
__device__ __forceinline__ double u52(uint32_t a, uint32_t b) {
    uint64_t m = (static_cast<uint64_t>(a >> 6) << 26) | static_cast<uint64_t>(b >> 6);
    return (static_cast<double>(m) + 0.5) * 0x1p-52;
}

__device__ __forceinline__ double stream_uniform(uint32_t k0, uint32_t k1, uint32_t tag, uint32_t step, uint32_t pid,
                                                 uint32_t draw) {
    uint32_t o[4];
    philox4x32_10(draw >> 1, pid, step, tag, k0, k1, o);
    return (draw & 1u) ? u52(o[2], o[3]) : u52(o[0], o[1]);
}

// Float uniform on the open interval from the top 23 bits of a Philox word:
// (w >> 9) * 2^-23 + 2^-24, built in the exponent-1 binade so no conversion
// instruction is issued.  (1 + k 2^-23) - (1 - 2^-24) is exact (Sterbenz).
__device__ __forceinline__ float u23(uint32_t w) {
    return __uint_as_float(0x3f800000u | (w >> 9)) - 0x1.fffffep-1f;
}

// The engine's per-particle stream: counter (draw >> 1, pid, step, tag).  The
// four words of the current Philox block are cached; a draw converts only the
// pair it uses.  rawf() reads the same draw as raw() rounded to the 2^-23 bin
// its high word selects, so the FP32 form follows the FP64 form's stream.
struct PhiloxRng {
    uint32_t k0, k1, tag, step, pid, draw;
    uint32_t block;
    uint32_t w[4];
    __device__ __forceinline__ void init(uint32_t kk0, uint32_t kk1, uint32_t t, uint32_t s, uint32_t p, uint32_t d) {
        k0 = kk0; k1 = kk1; tag = t; step = s; pid = p; draw = d; block = 0xffffffffu;
    }
    __device__ __forceinline__ void fetch() {
        uint32_t b = draw >> 1;
        if (b != block) {
            philox4x32_10(b, pid, step, tag, k0, k1, w);
            block = b;
        }
    }
    __device__ __forceinline__ double raw() {
        fetch();
        const bool odd = draw & 1u;
        const double u = u52(odd ? w[2] : w[0], odd ? w[3] : w[1]);
        ++draw;
        return u;
    }
    __device__ __forceinline__ float rawf() {
        fetch();
        float u = u23((draw & 1u) ? w[2] : w[0]);
        ++draw;
        return u;
    }
    // a draw whose value is not used
    __device__ __forceinline__ void skip() { ++draw; }
    // RadiationIMC::randomUnitOpen (radiation/RadiationIMC.hpp:700-713); a no-op on
    // these uniforms, kept for the shared code path.
    __device__ __forceinline__ double open() {
        double v = raw();
        return v <= 0.0 ? DBL_MIN : (v >= 1.0 ? ONE_BELOW : v);
    }
    __device__ __forceinline__ bool exhausted() const { return false; }
};

// The FP32-tracking form's per-particle stream: the same Philox counter
// (block, pid, step, tag) with all four words of a block used, one 23-bit float
// draw per word, so a collision and its isotropic re-scatter take under one
// block.  Draws the FP64 form consumes without using (the event-type draw)
// are not taken.  This stream is its own: the FP32 form's histories are
// statistically independent of the FP64 form's.
struct PhiloxRng4 {
    uint32_t k0, k1, tag, step, pid, draw;
    uint32_t block;
    uint32_t w[4];
    __device__ __forceinline__ void init(uint32_t kk0, uint32_t kk1, uint32_t t, uint32_t s, uint32_t p, uint32_t d) {
        k0 = kk0; k1 = kk1; tag = t; step = s; pid = p; draw = d; block = 0xffffffffu;
    }
    __device__ __forceinline__ float rawf() {
        const uint32_t b = draw >> 2;
        if (b != block) {
            philox4x32_10(b, pid, step, tag, k0, k1, w);
            block = b;
        }
        const uint32_t sel = draw & 3u;
        const uint32_t word = sel == 0 ? w[0] : (sel == 1 ? w[1] : (sel == 2 ? w[2] : w[3]));
        ++draw;
        return u23(word);
    }
    __device__ __forceinline__ void skip() {}
    __device__ __forceinline__ bool exhausted() const { return false; }
};

// Replay of a recorded tape of the reference's draws.
struct TapeRng {
    const double *tape;
    uint32_t len, pos;
    bool over;
    __device__ __forceinline__ double raw() {
        if (pos >= len) { over = true; return 0.5; }
        return tape[pos++];
    }
    __device__ __forceinline__ double open() {
        double v = raw();
        return v <= 0.0 ? DBL_MIN : (v >= 1.0 ? ONE_BELOW : v);
    }
    __device__ __forceinline__ float rawf() {
        return fminf(fmaxf(static_cast<float>(raw()), 0x1p-24f), 0x1.fffffep-1f);
    }
    __device__ __forceinline__ void skip() { (void)raw(); }
    __device__ __forceinline__ bool exhausted() const { return over; }
};

// ------------------------------------------------------------------ particle in registers
struct PartReg {
    double x, y, z, vx, vy, vz, t, w, w0;
    double nu;       // photon energy [erg] (multigroup)
    uint32_t cell;
};

__device__ __forceinline__ void cell_ijk(const Ctx &C, uint32_t c, uint32_t &i, uint32_t &j, uint32_t &k) {
    i = c % C.nx;
    uint32_t r = c / C.nx;
    j = r % C.ny;
    k = r / C.ny;
}

// STORM::fallback::abs (elementary/PointOps.hpp:71)
__device__ __forceinline__ double vnorm(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

// ------------------------------------------------------------------ Random Walk samplers (radiation/RandomWalk.hpp:81-137)
__device__ __forceinline__ double clampd(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }

__device__ inline double rw_sample_leak(const RwTables &T, double xi) {
    double target = 1.0 - xi;
    if (target >= T.surv[0]) return T.tau[0];
    if (target <= T.surv[RW_TABLE - 1]) return T.tau[RW_TABLE - 1];
    // std::lower_bound with comp(a, b) = a > b on the non-increasing survival
    // table: from the bucket's start, the first entry not above the target
    const int b = min(static_cast<int>(target * RW_LEAK_BUCKETS), RW_LEAK_BUCKETS - 1);
    uint32_t first = T.leakStart[b];
    while (first < RW_TABLE && T.surv[first] > target) ++first;
    if (first == 0) return T.tau[0];
    if (first == RW_TABLE) return T.tau[RW_TABLE - 1];
    double S0 = T.surv[first - 1], S1 = T.surv[first];
    double frac = (S0 - target) / (S0 - S1);
    double l0 = T.logTau[first - 1], l1 = T.logTau[first];
    double logT = l0 + frac * (l1 - l0);
    return exp(logT);
}

__device__ inline double rw_sample_radius(const RwTables &T, double tau, double xi) {
    double logTau = log(clampd(tau, 1e-8, 64.0));
    double tauPos = (logTau - T.logMin) / (T.logMax - T.logMin) * static_cast<double>(RW_TABLE - 1);
    uint32_t tauIdx = static_cast<uint32_t>(tauPos);
    if (tauIdx > RW_TABLE - 2) tauIdx = RW_TABLE - 2;
    double tauFrac = tauPos - static_cast<double>(tauIdx);
    double xiC = clampd(xi, 0.0, 1.0);
    double xiPos = xiC * static_cast<double>(RW_RADIUS - 1);
    uint32_t xiIdx = static_cast<uint32_t>(xiPos);
    if (xiIdx > RW_RADIUS - 2) xiIdx = RW_RADIUS - 2;
    double xiFrac = xiPos - static_cast<double>(xiIdx);
    const double *r0p = T.radius + static_cast<size_t>(tauIdx) * RW_RADIUS + xiIdx;
    const double *r1p = r0p + RW_RADIUS;
    double r00 = r0p[0], r01 = r0p[1], r10 = r1p[0], r11 = r1p[1];
    double r0 = r00 + xiFrac * (r01 - r00);
    double r1 = r10 + xiFrac * (r11 - r10);
    return clampd(r0 + tauFrac * (r1 - r0), 0.0, 1.0);
}

// ------------------------------------------------------------------ isotropic direction
// RadiationOpacityModel::isotropicVelocity (radiation/RadiationOpacityModel.hpp:139-150)
template <class RNG>
__device__ __forceinline__ void isotropic(RNG &rng, double c, double &vx, double &vy, double &vz) {
    double theta = TWO_PI_ISO * rng.raw();
    double cosTheta = 2.0 * rng.raw() - 1.0;
    double s2 = 1.0 - cosTheta * cosTheta;
    double sinTheta = sqrt(s2 > 0.0 ? s2 : 0.0);
    double st, ct;
    sincos(theta, &st, &ct);
    vx = sinTheta * ct * c;
    vy = sinTheta * st * c;
    vz = cosTheta * c;
}

// ------------------------------------------------------------------ tallies
// Sink for the two per-cell tallies a segment writes: the material energy
// (extensives[cell].internal_energy) and the time-integrated radiation energy
// (Erad_time_avg_[cell]).  LocalTally sums one segment's deposits (replay).
struct LocalTally {
    static constexpr bool kEg = false;   // no group time averages
    double mat_, rad_;
    double mx_, my_, mz_;   // momentum (moving material)
    __device__ __forceinline__ void mat(uint32_t, double v) { mat_ += v; }
    __device__ __forceinline__ void rad(uint32_t, double v) { rad_ += v; }
    __device__ __forceinline__ void mom(const struct Ctx &, uint32_t, double x, double y, double z) {
        mx_ += x; my_ += y; mz_ += z;
    }
};
// The transport kernels' tally: every segment adds its deposits to the cell with
// fire-and-forget atomics (RED) and counts itself for the per-cell segment
// counters.  (Summing a run of segments in one cell in registers first costs
// more in register spills than it saves in atomics.)
struct SegmentTally {
    static constexpr bool kEg = false;   // no group time averages
    double *eint, *erad;
    uint32_t *segs;        // NULL: no per-cell counters
    double depSum;
    __device__ __forceinline__ void init(double *e, double *a, uint32_t *sc) {
        eint = e; erad = a; segs = sc; depSum = 0.0;
    }
    __device__ __forceinline__ void enter(uint32_t c) { if (segs) atomicAdd(segs + c, 1u); }
    __device__ __forceinline__ void mat(uint32_t c, double v) { atomicAdd(eint + c, v); depSum += v; }
    __device__ __forceinline__ void rad(uint32_t c, double v) { atomicAdd(erad + c, v); }
    __device__ __forceinline__ void mom(const struct Ctx &C, uint32_t c, double x, double y, double z);
};
// The same with the group time averages (withEgTimeAvg): every Erad_time_avg
// contribution also goes to Eg_time_avg[cell][findGroup(frequency)] with the
// particle's lab frequency at that moment (radiation/RadiationIMC.hpp:1166-1172,
// 1485-1491, 1802-1808).  The kernels that take it are instantiated apart, so
// the others carry none of its code.
struct SegmentTallyEg : SegmentTally {
    static constexpr bool kEg = true;
    __device__ __forceinline__ void eg(const struct Ctx &C, uint32_t c, double v, double nu);
    __device__ __forceinline__ void eg32(const struct Ctx &C, uint32_t c, double v, float nu);
};

// Reproducible tallies: a value x (already multiplied by a power-of-two scale,
// |x| < 2^119) goes into four 30-bit limbs, high to low, each added with an
// integer atomic.  Integer addition is associative, so the sums do not depend on
// the order the segments arrive in; up to 2^33 contributions per cell fit in a
// limb's 64 bits.  Bits below the scale's unit are dropped, the same way in
// every run.  The limbs are split off the magnitude with exact floating-point
// steps (each remainder is a multiple of the value's unit in the last place
// and below the next power) and carry its sign.
__device__ __forceinline__ void fixed_add(unsigned long long *acc, uint32_t c, double x) {
    const double ax = fabs(x);
    const double h3 = floor(ax * 0x1p-90);
    const double r3 = ax - h3 * 0x1p90;
    const double h2 = floor(r3 * 0x1p-60);
    const double r2 = r3 - h2 * 0x1p60;
    const double h1 = floor(r2 * 0x1p-30);
    const double h0 = floor(r2 - h1 * 0x1p30);
    long long l3 = static_cast<long long>(h3), l2 = static_cast<long long>(h2), l1 = static_cast<long long>(h1),
              l0 = static_cast<long long>(h0);
    if (x < 0.0) { l3 = -l3; l2 = -l2; l1 = -l1; l0 = -l0; }
    unsigned long long *a = acc + 4 * static_cast<size_t>(c);
    if (l3) atomicAdd(a + 3, static_cast<unsigned long long>(l3));
    if (l2) atomicAdd(a + 2, static_cast<unsigned long long>(l2));
    if (l1) atomicAdd(a + 1, static_cast<unsigned long long>(l1));
    if (l0) atomicAdd(a, static_cast<unsigned long long>(l0));
}
// The value of a cell's four limbs after the carries are propagated (integer
// arithmetic, then one fixed sequence of floating-point operations).
__device__ __forceinline__ double fixed_value(const unsigned long long *acc, uint32_t c) {
    const unsigned long long *a = acc + 4 * static_cast<size_t>(c);
    long long v0 = static_cast<long long>(a[0]), v1 = static_cast<long long>(a[1]), v2 = static_cast<long long>(a[2]),
              v3 = static_cast<long long>(a[3]);
    long long k = v0 >> 30; v0 -= k * (1ll << 30); v1 += k;
    k = v1 >> 30; v1 -= k * (1ll << 30); v2 += k;
    k = v2 >> 30; v2 -= k * (1ll << 30); v3 += k;
    return ((static_cast<double>(v3) * 0x1p90 + static_cast<double>(v2) * 0x1p60) + static_cast<double>(v1) * 0x1p30) +
           static_cast<double>(v0);
}
// The transport tally with reproducible sums (kernels of their own, as for the
// group time averages): the same calls, fixed-point limbs instead of FP64 atomics.
struct SegmentTallyFixed : SegmentTally {
    static constexpr bool kEg = false;
    unsigned long long *fm, *fr;
    double sm, sr;
    __device__ __forceinline__ void init_fixed(const struct Ctx &C);
    __device__ __forceinline__ void mat(uint32_t c, double v) { fixed_add(fm, c, v * sm); depSum += v; }
    __device__ __forceinline__ void rad(uint32_t c, double v) { fixed_add(fr, c, v * sr); }
};

// ------------------------------------------------------------------ multigroup
// planck_integral(a, b) = 15/pi^4 int_a^b x^3/(e^x - 1) dx from Clark's two
// published series: the Bernoulli expansion below x = 0.5 and the exponential
// tail series sum_n e^{-n x} (x^3/n + 3x^2/n^2 + 6x/n^3 + 6/n^4) above, with the
// host table build's switch point and stopping rule.  On the device the tail's
// exponentials come by recurrence, e^{-(n+1)x} = e^{-nx} e^{-x}, and each term
// takes one division; both change the sum by about n ulps (n < 100 terms
// where x >= 0.5), far inside the 1e-12 the tables are held to.
constexpr double PI_NORM_PI = 3.14159265358979323846;
__device__ __forceinline__ double pi_norm() { return 15.0 / (PI_NORM_PI * PI_NORM_PI * PI_NORM_PI * PI_NORM_PI); }
// The series' constants, folded at compile time so that the device multiplies
// instead of dividing: the small-x coefficients B_k / (k! (k + 3)), and 1/n^j
// (j = 1..4) for the first PI_TAIL_TABLE tail terms.  Both change the sums by
// a few ulps, inside the tables' 1e-12.
struct PiSmallCoef {
    double c[21];
    constexpr PiSmallCoef() : c() {
        const double B[21] = {1.0, -0.5, 1.0 / 6.0, 0.0, -1.0 / 30.0, 0.0, 1.0 / 42.0, 0.0, -1.0 / 30.0, 0.0,
                              5.0 / 66.0, 0.0, -691.0 / 2730.0, 0.0, 7.0 / 6.0, 0.0, -3617.0 / 510.0, 0.0,
                              43867.0 / 798.0, 0.0, -174611.0 / 330.0};
        double fact = 1.0;
        for (int k = 0; k <= 20; ++k) {
            if (k > 0) fact *= k;
            c[k] = B[k] / (fact * (k + 3));
        }
    }
};
constexpr int PI_TAIL_TABLE = 128;
struct PiTailInv {
    double v[4 * PI_TAIL_TABLE];   // per n: 1/n, 1/n^2, 1/n^3, 1/n^4
    constexpr PiTailInv() : v() {
        for (int n = 1; n <= PI_TAIL_TABLE; ++n) {
            const double d = n, d2 = d * d;
            v[4 * (n - 1)] = 1.0 / d;
            v[4 * (n - 1) + 1] = 1.0 / d2;
            v[4 * (n - 1) + 2] = 1.0 / (d2 * d);
            v[4 * (n - 1) + 3] = 1.0 / (d2 * d2);
        }
    }
};
static __constant__ PiSmallCoef c_piSmall = PiSmallCoef();
static __constant__ PiTailInv c_piTail = PiTailInv();

__device__ inline double pi_small_series(double x) {
    // x^3 sum_k c_k x^k, the zero coefficients skipped, by Horner in x
    double sum = c_piSmall.c[20];
#pragma unroll
    for (int k = 19; k >= 0; --k) sum = sum * x + c_piSmall.c[k];
    return sum * (x * x * x);
}
__device__ inline double pi_tail_series(double x) {
    const double e1 = exp(-x);
    const double x2 = x * x, x3 = x2 * x;
    const double a2 = 3.0 * x2, a3 = 6.0 * x;
    double sum = 0.0, e = e1;
    const double e1sq = e1 * e1;
    // every lane of a warp takes term n at the same time, so the table read is
    // uniform; terms go in pairs, whose exponentials are two independent
    // products, and the sum adds them in order
    int n = 1;
    for (; n + 1 <= PI_TAIL_TABLE && e != 0.0; n += 2) {
        const double *iv = c_piTail.v + 4 * (n - 1);
        const double eb = e * e1;
        const double ta = e * (((x3 * iv[0] + a2 * iv[1]) + a3 * iv[2]) + 6.0 * iv[3]);
        const double tb = eb * (((x3 * iv[4] + a2 * iv[5]) + a3 * iv[6]) + 6.0 * iv[7]);
        sum += ta;
        if (ta < 1e-18 * sum) return sum;
        sum += tb;
        if (tb < 1e-18 * sum) return sum;
        e *= e1sq;
    }
    for (; n < 100000 && e != 0.0; ++n) {
        const double dn = n;
        const double d2 = dn * dn;
        const double term = e * ((((x3 * dn + a2) * dn + a3) * dn + 6.0) / (d2 * d2));
        sum += term;
        if (term < 1e-18 * sum) break;
        e *= e1;
    }
    return sum;
}
// One group bound's share of planck_integral: the tail sum where x >= 0.5 and
// the cumulative 15/pi^4 int_0^x.  A table over G groups evaluates each of its
// G + 1 bounds once instead of twice.
struct PiBound {
    double x, tail, cum;
};
__device__ inline PiBound pi_bound(double x) {
    PiBound r{x, 0.0, 0.0};
    if (!(x > 0.0)) return r;
    if (x < 0.5) {
        r.cum = pi_norm() * pi_small_series(x);
    } else {
        r.tail = pi_tail_series(x);
        r.cum = 1.0 - pi_norm() * r.tail;
    }
    return r;
}
// planck_integral(a, b) from its two bounds (a > 0, b > a)
__device__ __forceinline__ double pi_between(const PiBound &a, const PiBound &b) {
    if (a.x >= 0.5 && b.x >= 0.5) return pi_norm() * (a.tail - b.tail);
    return b.cum - a.cum;
}
__device__ inline double planck_integral(double a, double b) { return pi_between(pi_bound(a), pi_bound(b)); }

// std::clamp(nu, b_0, b_G) (RadiationIMC::clampFrequencyToBounds, radiation/RadiationIMC.hpp:869-872)
__device__ __forceinline__ double mg_clamp(const Ctx &C, double nu) {
    const double lo = C.gb[0], hi = C.gb[C.groups];
    return nu < lo ? lo : (hi < nu ? hi : nu);
}
// RadiationOpacityModel::findGroup (radiation/RadiationOpacityModel.hpp:76-86):
// the first g with nu < b_{g+1}, else the last group
__device__ __forceinline__ uint32_t mg_find_group(const Ctx &C, double nu) {
    uint32_t lo = 0, hi = C.groups - 1;   // answer in [lo, hi]
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (nu < C.gb[mid + 1]) hi = mid; else lo = mid + 1;
    }
    return lo;
}
__device__ __forceinline__ void SegmentTallyFixed::init_fixed(const Ctx &C) {
    fm = C.fixMat; fr = C.fixRad; sm = C.fixScaleMat; sr = C.fixScaleRad;
}
__device__ __forceinline__ void SegmentTallyEg::eg(const Ctx &C, uint32_t c, double v, double nu) {
    atomicAdd(C.egAvg + static_cast<size_t>(c) * C.groups + mg_find_group(C, nu), v);
}
// kT of the opacity model: k_B max(T, 1 K)
__device__ __forceinline__ double mg_kT(const Ctx &C, uint32_t c) {
    const double T = C.T[c];
    return C.kBoltz * (T < 1.0 ? 1.0 : T);
}
// (1 - e^{-E/kT})^s
__device__ __forceinline__ double mg_stim(const Ctx &C, double E, double kT) {
    const double x = -expm1(-E / kT);
    return C.mgS == 1.0 ? x : pow(x, C.mgS);
}
// sigma0 / ((kT)^q E^p) (1 - e^{-E/kT})^s with (kT)^q = kTq and E^p = Ep given
__device__ __forceinline__ double mg_sigma(const Ctx &C, uint32_t c, double E, double kT, double kTq, double Ep) {
    double v = C.sig0[c] / (kTq * Ep);
    if (C.mgS != 0.0) v *= mg_stim(C, E, kT);
    return v;
}
// CalcAbsorptionOpacity(cell, frequency); (kT)^q comes from the cell's prestep
// value, E^p from the per-group table when the opacity is taken at the group centre
__device__ __forceinline__ double mg_absorption(const Ctx &C, uint32_t c, double nu) {
    const double kT = mg_kT(C, c);
    if (C.mgGroupConst) {
        const uint32_t g = mg_find_group(C, nu);
        return mg_sigma(C, c, 0.5 * (C.gb[g] + C.gb[g + 1]), kT, C.mgKTq[c], C.mgEp[g]);
    }
    const double E = nu < C.gb[0] ? C.gb[0] : nu;
    return mg_sigma(C, c, E, kT, C.mgKTq[c], pow(E, C.mgP));
}
// GetThermalEnergy (examples/densmore2012/DensmoreOpacity.hpp:71-82): the
// inverse of the cell's cumulative sigma_g B_g by STORM::LinearInterpolation
// (utils/LinearInterpolation.hpp:18-42); the base class's uniform draw when the
// spectrum is empty.  Returns a negative energy where LinearInterpolation
// throws (x beyond the table).
__device__ inline double mg_thermal_energy(const Ctx &C, uint32_t c, double random) {
    const uint32_t G = C.groups;
    const double *x = C.mgCdf + static_cast<size_t>(c) * (G + 1);
    const double *y = C.gb;
    const double total = x[G];
    if (!(total > 0.0) || !isfinite(total)) return y[0] + random * (y[G] - y[0]);
    const double r = isfinite(random) ? (random < 0.0 ? 0.0 : (ONE_BELOW < random ? ONE_BELOW : random)) : 0.5;
    const double xi = r * total;
    // std::upper_bound: the first x > xi
    uint32_t first = 0, count = G + 1;
    while (count > 0) {
        const uint32_t step = count >> 1, it = first + step;
        if (!(xi < x[it])) { first = it + 1; count -= step + 1; } else count = step;
    }
    if (first == G + 1) return fabs(x[G] - xi) < 1e-12 ? y[G] : -1.0;
    if (fabs(x[first] - xi) < 1e-12 || first == 0) return y[first];
    return y[first] + (xi - x[first]) * (y[first - 1] - y[first]) / (x[first - 1] - x[first]);
}

// ------------------------------------------------------------------ Random Walk jump
// RadiationIMC::tryRandomWalkStep (radiation/RadiationIMC.hpp:1065-1276), gray.
// Returns -1 when the walk is not taken (no draws consumed), else a ParticleStatus.
// A cell's faces as computeMinDistanceToFaces and the Random Walk's shrink loop
// see them: ScalarProd(location - facePoint, inwardNormal) per face in
// GetCellFaces order, and the mesh point the nudges aim at.  On a Cartesian
// cell the inward normals are exact unit vectors, so each product reduces
// exactly to one coordinate difference.
struct CartGeom {
    double xl, xh, yl, yh, zl, zh, cx, cy, cz;
    __device__ __forceinline__ int nf() const { return 6; }
    __device__ __forceinline__ double dist(int s, double x, double y, double z) const {
        switch (s) {
        case 0: return x - xl;
        case 1: return xh - x;
        case 2: return y - yl;
        case 3: return yh - y;
        case 4: return z - zl;
        default: return zh - z;
        }
    }
};
struct PolyGeom {
    const Ctx *C;
    uint32_t k0, k1;
    double cx, cy, cz;
    __device__ __forceinline__ int nf() const { return static_cast<int>(k1 - k0); }
    __device__ __forceinline__ double dist(int s, double x, double y, double z) const {
        const double4 n = C->cfN[k0 + s], q = C->cfP[k0 + s];
        return (x - q.x) * n.x + (y - q.y) * n.y + (z - q.z) * n.z;
    }
};

// ------------------------------------------------------------------ moving material
__device__ __forceinline__ void SegmentTally::mom(const Ctx &C, uint32_t c, double x, double y, double z) {
    double *m = C.mom + 3 * static_cast<size_t>(c);
    atomicAdd(m, x);
    atomicAdd(m + 1, y);
    atomicAdd(m + 2, z);
}

// computeDopplerShift (radiation/RadiationIMC.hpp:228-245): the lab-to-comoving
// factor gamma (1 - v.u / c^2) for a particle of lab velocity u in a cell
// moving at v; 1 for a cell at rest.
__device__ __forceinline__ double doppler_shift(const Ctx &C, const double4 &v, double ux, double uy, double uz) {
    const double v2 = (v.x * v.x + v.y * v.y) + v.z * v.z;
    if (v2 < 1e-30) return 1.0;
    const double gamma = 1.0 / sqrt(1.0 - v2 * C.invC2);
    return gamma * (1.0 - ((v.x * ux + v.y * uy) + v.z * uz) * C.invC2);
}

// lorentzTransformToLab (radiation/RadiationIMC.hpp:286-310): a comoving
// particle to the lab frame -- frequency and weight by the Doppler factor of
// the reversed cell velocity, the direction boosted and renormalised to c.
__device__ __forceinline__ void lorentz_to_lab(const Ctx &C, const double4 &v, PartReg &p) {
    const double v2 = (v.x * v.x + v.y * v.y) + v.z * v.z;
    if (v2 < 1e-30) return;
    const double gamma = 1.0 / sqrt(1.0 - C.invC2 * v2);
    const double nx = v.x * (-1.0), ny = v.y * (-1.0), nz = v.z * (-1.0);
    const double shift = gamma * (1.0 - ((nx * p.vx + ny * p.vy) + nz * p.vz) * C.invC2);
    p.nu *= shift;
    p.w *= shift;
    const double vDotP = (p.vx * nx + p.vy * ny) + p.vz * nz;
    const double k = (gamma - 1.0) * vDotP / v2 - gamma;
    p.vx = p.vx + nx * k;
    p.vy = p.vy + ny * k;
    p.vz = p.vz + nz * k;
    const double speed = vnorm(p.vx, p.vy, p.vz);
    if (speed > 0.0) {
        const double f = C.clight / speed;
        p.vx = p.vx * f;
        p.vy = p.vy * f;
        p.vz = p.vz * f;
    }
}

// extensives_[cell].momentum += (w0 u0 - w u) / c^2 (the momentum a scatter or
// a Random Walk jump leaves in the cell)
template <class TALLY>
__device__ __forceinline__ void momentum_exchange(const Ctx &C, TALLY &tal, uint32_t cell, double w0, double ux0,
                                                  double uy0, double uz0, const PartReg &p) {
    tal.mom(C, cell, (w0 * ux0 - p.w * p.vx) * C.invC2, (w0 * uy0 - p.w * p.vy) * C.invC2,
            (w0 * uz0 - p.w * p.vz) * C.invC2);
}

template <bool MGP, class GEOM, class RNG, class TALLY, bool HYDRO = false>
__device__ inline int try_random_walk(const Ctx &C, PartReg &p, RNG &rng, TALLY &tal, const double4 &cp,
                                      const GEOM &g) {
    const uint32_t cell = p.cell;
    const double cx = g.cx, cy = g.cy, cz = g.cz;
    // computeMinDistanceToFaces (:956-969) in GetCellFaces order
    double Ro = DBL_MAX;
    for (int s = 0; s < g.nf(); ++s) {
        const double d = g.dist(s, p.x, p.y, p.z);
        Ro = (d < Ro) ? d : Ro;
    }
    Ro = (Ro > 0.0) ? Ro : 0.0;
    const double c = C.clight;
    const bool pgrw = MGP && C.groups >= 2;
    double sigmaT, sigmaAeff, Dphys, gammaRw = 1.0;
    uint32_t cutoff = 0;
    if (pgrw) {   // PGRW cell data (:1080-1087)
        const double4 g4 = C.pgrw[cell];
        sigmaT = g4.x; sigmaAeff = g4.y; Dphys = g4.z; gammaRw = g4.w;
        cutoff = C.pgrwCut[cell];
    } else {
        sigmaT = C.rwSigT[cell];
        sigmaAeff = C.sigA[cell];
        Dphys = cp.w;
    }
    bool doRW = (Ro > 0.0 && sigmaT > 0.0 && Dphys > 0.0 && Ro * sigmaT >= C.rwMinParticle);
    // (:1098-1115): the (comoving) frequency against the cutoff.  The static
    // form keeps its own one-line test: the moving-material form of it, even
    // where it reduces to the same operations, changed the compiled kernel's
    // layout and cost the multigroup FP64 transport a quarter of its speed
    // through instruction-fetch stalls (measured with ncu).
    if constexpr (HYDRO) {
        if (doRW && pgrw) {
            double coFreq = p.nu;
            if (C.withHydro) coFreq *= doppler_shift(C, C.vel[cell], p.vx, p.vy, p.vz);
            if (mg_clamp(C, coFreq) >= C.gb[cutoff]) doRW = false;
        }
    } else {
        if (doRW && pgrw && mg_clamp(C, p.nu) >= C.gb[cutoff]) doRW = false;
    }
    if (!doRW) return -1;
    struct { double vx, vy, vz, w; } old{};   // (:1121-1122), moving material only
    if constexpr (HYDRO) { old.vx = p.vx; old.vy = p.vy; old.vz = p.vz; old.w = p.w; }
    const double fl = pgrw ? C.fleck[cell] : 0.0;
    double tauLeak = rw_sample_leak(C.rw, rng.open());
    double tLeak = tauLeak * Ro * Ro / Dphys;
    double tCensus = p.t;
    double tUp = DBL_MAX;   // upscatter out of the diffusive groups (:1130-1135)
    if (pgrw && gammaRw < 1.0 && sigmaAeff > 0.0 && fl > 0.0) {
        double xiUp = rng.open();
        tUp = -log(xiUp) / (c * (1.0 - fl) * sigmaAeff * (1.0 - gammaRw));
    }
    int ev;
    double dt;
    if (tLeak <= tCensus && tLeak <= tUp) { ev = 0; dt = tLeak; }
    else if (tCensus <= tUp) { ev = 1; dt = tCensus; }
    else { ev = 2; dt = tUp; }
    const double rate = pgrw ? sigmaAeff * fl * c : cp.y;   // sigma_a_eff * f * c
    double rwExp = expm1(-dt * rate);
    if (!C.noFeedback) tal.mat(cell, -rwExp * p.w);
    if (rate > 0.0) tal.rad(cell, p.w * rwExp * (pgrw ? (-1.0 / rate) : cp.z));
    if constexpr (TALLY::kEg) {
        if (rate > 0.0) tal.eg(C, cell, p.w * rwExp * (pgrw ? (-1.0 / rate) : cp.z), p.nu);
    }
    p.w *= 1.0 + rwExp;
    p.t -= dt;
    if (fabs(p.w) < p.w0 * 1e-4) {
        if (!C.noFeedback) tal.mat(cell, p.w);
        return REMOVE;
    }
    double cosTheta = 2.0 * rng.open() - 1.0;
    double s2 = 1.0 - cosTheta * cosTheta;
    double sinTheta = sqrt(s2 > 0.0 ? s2 : 0.0);
    double phi = 2.0 * RW_PI * rng.open();
    double sphi, cphi;
    sincos(phi, &sphi, &cphi);
    double dx = sinTheta * cphi, dy = sinTheta * sphi, dz = cosTheta;
    double disp;
    if (ev == 0) disp = Ro;
    else {
        double tauPos = Dphys * dt / (Ro * Ro);
        disp = Ro * rw_sample_radius(C.rw, tauPos, rng.open());
    }
    if (disp > Ro * (1.0 + 1e-12)) disp = Ro;
    const double ox = p.x, oy = p.y, oz = p.z;
    double lx = ox + disp * dx, ly = oy + disp * dy, lz = oz + disp * dz;
    lx = lx * (1.0 - RW_NUDGE) + RW_NUDGE * cx;
    ly = ly * (1.0 - RW_NUDGE) + RW_NUDGE * cy;
    lz = lz * (1.0 - RW_NUDGE) + RW_NUDGE * cz;
    // shrink until inside every face plane (:1216-1228)
    int guard = 0;
    for (int s = 0; s < g.nf(); ++s) {
        const double q = g.dist(s, lx, ly, lz);
        if (q < 0.0) {
            disp *= 0.99;
            lx = ox + disp * dx;
            ly = oy + disp * dy;
            lz = oz + disp * dz;
            s = -1;
            if (++guard > RW_SHRINK_CAP) return -2;
        }
    }
    p.x = lx; p.y = ly; p.z = lz;
    isotropic(rng, c, p.vx, p.vy, p.vz);
    if (ev == 2) {   // upscatter: a frequency above the cutoff from the emission spectrum (:1232-1250)
        const double *cdf = C.mgCdf + static_cast<size_t>(cell) * (C.groups + 1);
        const double cdfAtCutoff = cdf[cutoff], cdfTotal = cdf[C.groups];
        if (cdfTotal > cdfAtCutoff) {
            double lo = cdfAtCutoff / cdfTotal;
            double xi = rng.open();
            p.nu = mg_thermal_energy(C, cell, lo + xi * (1.0 - lo));
        } else {
            p.nu = nextafter(C.gb[cutoff], DBL_MAX);
        }
        p.nu = mg_clamp(C, p.nu);
    }
    if constexpr (HYDRO) {
        if (C.withHydro) {   // the comoving jump's end back to the lab frame (:1252-1268)
            lorentz_to_lab(C, C.vel[cell], p);
            if (pgrw) p.nu = mg_clamp(C, p.nu);
            if (!C.noFeedback) momentum_exchange(C, tal, cell, old.w, old.vx, old.vy, old.vz, p);
        }
    }
    return (ev == 1) ? DONE : NO_CELL_MOVE;
}

// ------------------------------------------------------------------ physics step
// tryDDMCStep's leak face (radiation/RadiationIMC.hpp:1524-1540): subtract the
// positive face rates in GetCellFaces order from u * total; the last face
// with a rate when rounding leaves some over; -1 when no face has one.
template <class RNG>
__device__ __forceinline__ int ddmc_pick_face(RNG &rng, const double *rates, int nf, double total) {
    double facePick = rng.open() * total;
    int chosen = -1, last = -1;
    for (int s = 0; s < nf; ++s) {
        const double r = rates[s];
        if (!(r > 0.0) || chosen >= 0) continue;
        last = s;
        facePick -= r;
        if (facePick <= 0.0) chosen = s;
    }
    return chosen < 0 ? last : chosen;
}
// tryDDMCStep's leak direction (:1561-1589): cosine law about the unit normal n
// (pointing at the neighbour), in the frame of a helper axis.
template <class RNG>
__device__ __forceinline__ void ddmc_leak_direction(RNG &rng, const double n[3], double dir[3]) {
    const double PI_D = 3.14159265358979323846;
    const double u4 = rng.open();
    const double xiMu = (u4 < 1.0) ? u4 : 1.0;   // std::min(1.0, u)
    const double mu = sqrt(xiMu);
    const double phiLeak = 2.0 * PI_D * rng.open();
    const double st2 = 1.0 - mu * mu;
    const double sinTheta = sqrt(st2 > 0.0 ? st2 : 0.0);
    double h[3] = {0.0, 0.0, 0.0};
    if (fabs(n[0]) < 0.9) h[0] = 1.0; else h[1] = 1.0;
    const double hn = h[0] * n[0] + h[1] * n[1] + h[2] * n[2];
    double e1[3] = {h[0] - n[0] * hn, h[1] - n[1] * hn, h[2] - n[2] * hn};
    const double e1m = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    if (e1m > 0.0) { e1[0] = e1[0] / e1m; e1[1] = e1[1] / e1m; e1[2] = e1[2] / e1m; }
    double e2[3] = {n[1] * e1[2] - n[2] * e1[1], n[2] * e1[0] - n[0] * e1[2], n[0] * e1[1] - n[1] * e1[0]};
    const double e2m = sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    if (e2m > 0.0) { e2[0] = e2[0] / e2m; e2[1] = e2[1] / e2m; e2[2] = e2[2] / e2m; }
    const double a1 = sinTheta * cos(phiLeak), a2 = sinTheta * sin(phiLeak);
#pragma unroll
    for (int q = 0; q < 3; ++q) dir[q] = (n[q] * mu + e1[q] * a1) + e2[q] * a2;
    const double dm = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    if (dm > 0.0) { dir[0] = dir[0] / dm; dir[1] = dir[1] / dm; dir[2] = dir[2] / dm; }
}

// RadiationIMC::tryDDMCStep (radiation/RadiationIMC.hpp:1416-1612) on a
// Cartesian cell.  Returns -1 when the step is not taken (no draws consumed),
// else the ParticleStatus; a leak sets face and next.  precomputeDDMCData sets
// gamma = 1 in both of its branches, so the upscatter rate is always zero and
// every event that is not census leaks through a face.
template <class RNG, class TALLY>
__device__ inline int try_ddmc(const Ctx &C, PartReg &p, RNG &rng, TALLY &tal, double xl, double xh, double yl,
                               double yh, double zl, double zh, int &face, uint32_t &next) {
    const uint32_t cell = p.cell;
    const double total = C.ddmcTot[cell];
    if (!(total > 0.0)) return -1;
    const double4 dd = C.ddmc[cell];   // sigma_T, sigma_A, -, D
    double d[6] = {p.x - xl, xh - p.x, p.y - yl, yh - p.y, p.z - zl, zh - p.z};
    double Ro = DBL_MAX;
#pragma unroll
    for (int s = 0; s < 6; ++s) Ro = (d[s] < Ro) ? d[s] : Ro;
    Ro = (Ro > 0.0) ? Ro : 0.0;
    if (Ro * dd.x < C.ddmcMinParticle) return -1;
    if (C.ddmcPgrw) {
        const uint32_t cut = C.ddmcCut[cell];
        if (cut == 0 || cut > C.groups) return -1;
        if (mg_clamp(C, p.nu) >= C.gb[cut]) return -1;
    }
    const double f = C.fleck[cell];
    const double eventRate = total;
    const double tEvent = -log(rng.open()) / eventRate;
    const double tCensus = p.t;
    const double dt = (tCensus < tEvent) ? tCensus : tEvent;   // std::min(tEvent, tCensus)
    const bool censusEvent = (tCensus <= tEvent);
    const double absRate = dd.y * f * C.clight;
    const double oldWeight = p.w;
    const double expFactor = expm1(-dt * absRate);
    if (!C.noFeedback) tal.mat(cell, -expFactor * oldWeight);
    const double integrated = (absRate > 0.0) ? oldWeight * expFactor * (-1.0 / absRate) : oldWeight * dt;
    tal.rad(cell, integrated);
    if constexpr (TALLY::kEg) tal.eg(C, cell, integrated, p.nu);
    p.w *= 1.0 + expFactor;
    p.t -= dt;
    if (fabs(p.w) < p.w0 * 1e-3) {
        if (!C.noFeedback) tal.mat(cell, p.w);
        return REMOVE;
    }
    if (censusEvent) return DONE;
    const double eventPick = rng.open() * eventRate;
    if (!(eventPick <= total)) return DONE;   // the upscatter branch; unreachable with a zero upscatter rate
    // the leak face: subtract the face rates in GetCellFaces order
    const int chosen = ddmc_pick_face(rng, C.ddmcRate + static_cast<size_t>(cell) * 6, 6, total);
    if (chosen < 0) return DONE;
    uint32_t i, j, k;
    cell_ijk(C, cell, i, j, k);
    const int axis = chosen >> 1, hi = chosen & 1;
    // FaceCM: the face plane's coordinate, the cell's centre along the other axes
    double fc[3] = {C.xc[i], C.yc[j], C.zc[k]};
    fc[axis] = (axis == 0) ? (hi ? xh : xl) : (axis == 1 ? (hi ? yh : yl) : (hi ? zh : zl));
    // Normal(face) is the +axis unit vector; flipped to point at the neighbour
    double n[3] = {axis == 0 ? 1.0 : 0.0, axis == 1 ? 1.0 : 0.0, axis == 2 ? 1.0 : 0.0};
    if (!hi) { n[0] = n[0] * (-1.0); n[1] = n[1] * (-1.0); n[2] = n[2] * (-1.0); }
    double dir[3];
    ddmc_leak_direction(rng, n, dir);
    p.x = fc[0]; p.y = fc[1]; p.z = fc[2];
    p.vx = dir[0] * C.clight; p.vy = dir[1] * C.clight; p.vz = dir[2] * C.clight;
    face = chosen;
    switch (chosen) {
    case 0: next = cell - 1; break;
    case 1: next = cell + 1; break;
    case 2: next = cell - C.nx; break;
    case 3: next = cell + C.nx; break;
    case 4: next = cell - C.nx * C.ny; break;
    default: next = cell + C.nx * C.ny; break;
    }
    return CELL_MOVE;
}

// tryDDMCStep on a convex-polyhedral cell: the distances to the faces, the
// leak face and its neighbour from the cell-face slots; the particle leaves
// from the face centroid (FaceCM) along a cosine law about Normal(face) / |.|
// turned toward the neighbour's mesh point.  The inward slot normal is that
// unit normal up to its sign, so negating it and applying the same test gives
// the reference's vector.  Gray only (polyhedral meshes take no multigroup
// opacity).
template <class RNG, class TALLY>
__device__ inline int try_ddmc_poly(const Ctx &C, PartReg &p, RNG &rng, TALLY &tal, const PolyGeom &g,
                                    uint32_t &next) {
    const uint32_t cell = p.cell;
    const double total = C.ddmcTot[cell];
    if (!(total > 0.0)) return -1;
    const double4 dd = C.ddmc[cell];   // sigma_T, sigma_A, -, D
    double Ro = DBL_MAX;
    for (int s = 0; s < g.nf(); ++s) {
        const double d = g.dist(s, p.x, p.y, p.z);
        Ro = (d < Ro) ? d : Ro;
    }
    Ro = (Ro > 0.0) ? Ro : 0.0;
    if (Ro * dd.x < C.ddmcMinParticle) return -1;
    const double f = C.fleck[cell];
    const double eventRate = total;
    const double tEvent = -log(rng.open()) / eventRate;
    const double tCensus = p.t;
    const double dt = (tCensus < tEvent) ? tCensus : tEvent;   // std::min(tEvent, tCensus)
    const bool censusEvent = (tCensus <= tEvent);
    const double absRate = dd.y * f * C.clight;
    const double oldWeight = p.w;
    const double expFactor = expm1(-dt * absRate);
    if (!C.noFeedback) tal.mat(cell, -expFactor * oldWeight);
    const double integrated = (absRate > 0.0) ? oldWeight * expFactor * (-1.0 / absRate) : oldWeight * dt;
    tal.rad(cell, integrated);
    p.w *= 1.0 + expFactor;
    p.t -= dt;
    if (fabs(p.w) < p.w0 * 1e-3) {
        if (!C.noFeedback) tal.mat(cell, p.w);
        return REMOVE;
    }
    if (censusEvent) return DONE;
    const double eventPick = rng.open() * eventRate;
    if (!(eventPick <= total)) return DONE;   // the upscatter branch; unreachable with a zero upscatter rate
    const int chosen = ddmc_pick_face(rng, C.ddmcRate + g.k0, g.nf(), total);
    if (chosen < 0) return DONE;
    const uint32_t k = g.k0 + static_cast<uint32_t>(chosen);
    const uint32_t nb = C.cfNext[k];
    const double4 nin = C.cfN[k], fcm = C.cfP[k];
    double n[3] = {nin.x * (-1.0), nin.y * (-1.0), nin.z * (-1.0)};
    const double tx = C.mpx[nb] - C.mpx[cell], ty = C.mpy[nb] - C.mpy[cell], tz = C.mpz[nb] - C.mpz[cell];
    if (n[0] * tx + n[1] * ty + n[2] * tz < 0.0) { n[0] = n[0] * (-1.0); n[1] = n[1] * (-1.0); n[2] = n[2] * (-1.0); }
    double dir[3];
    ddmc_leak_direction(rng, n, dir);
    p.x = fcm.x; p.y = fcm.y; p.z = fcm.z;
    p.vx = dir[0] * C.clight; p.vy = dir[1] * C.clight; p.vz = dir[2] * C.clight;
    next = nb;
    return CELL_MOVE;
}

struct PhysOut {
    int status;        // ParticleStatus or -1 error code in errCode
    int face;          // crossed side (GetCellFaces order) for CELL_MOVE
    uint32_t next;     // neighbour cell or OUTSIDE (face crossings)
    uint32_t ghost;    // Ncells + global face index when next is OUTSIDE
    int usedRW;
    int errCode;
};

// global face index of side s of cell (i,j,k) (the grid's face numbering)
__device__ __forceinline__ uint32_t face_index(const Ctx &C, uint32_t i, uint32_t j, uint32_t k, int s) {
    uint32_t nx = C.nx, ny = C.ny, nz = C.nz;
    uint32_t nxf = (nx + 1) * ny * nz, nyf = nx * (ny + 1) * nz;
    switch (s) {
    case 0: return i + (nx + 1) * (j + ny * k);
    case 1: return (i + 1) + (nx + 1) * (j + ny * k);
    case 2: return nxf + i + nx * (j + (ny + 1) * k);
    case 3: return nxf + i + nx * ((j + 1) + (ny + 1) * k);
    case 4: return nxf + nyf + i + nx * (j + ny * k);
    default: return nxf + nyf + i + nx * (j + ny * (k + 1));
    }
}

// Per-cell constants of a segment, evaluated once per step with the same
// operations the reference evaluates per segment, so the values are identical:
//   x = scatteringLength = 1 / (sigma_s + (1 - f) sigma_a)  (+inf when that is <= 0)
//   y = tmp2 = sigma_a * f * c  (also the Random Walk absorption rate)
//   z = -1 / tmp2
//   w = D = c / (3 sigma_T) for the Random Walk (0 when sigma_T <= 0)
__device__ __forceinline__ double4 cell_phys(double sigA, double sigS, double f, double sigT, double c) {
    const double eventOpacity = sigS + (1.0 - f) * sigA;
    double4 r;
    r.x = (eventOpacity > 0.0) ? 1.0 / eventOpacity : CUDART_INF;
    r.y = sigA * f * c;
    r.z = -1.0 / r.y;
    r.w = (sigT > 0.0) ? c / (3.0 * sigT) : 0.0;
    return r;
}

// A particle being tracked: its state plus the cell coordinates and speed kept
// in registers between segments.
struct Track {
    PartReg p;
    uint32_t i, j, k;
    double speed;   // STORM::fallback::abs(velocity), recomputed when the velocity changes
};

__device__ __forceinline__ void track_begin(const Ctx &C, Track &T) {
    cell_ijk(C, T.p.cell, T.i, T.j, T.k);
    T.speed = vnorm(T.p.vx, T.p.vy, T.p.vz);
}

// RadiationIMC::step (radiation/RadiationIMC.hpp:1700-1881), gray, without hydro,
// including the face search of Particle::distanceToNearestFace
// (particle/Particle.hpp:188-279).  For an axis-aligned cell the inward normals
// are exact +-unit vectors, so (p_f - x).n and n.v reduce exactly to one
// coordinate difference and one velocity component, and each axis offers at
// most one candidate face.  The candidates are ordered by comparing
// |n_a| |v_b| with |n_b| |v_a| (no division), and only the winner's exit time
// is divided out: that time is bit-identical to the reference's; the choice of
// face can differ only when two exit times agree to within rounding.
//
// FULL compiles the multigroup and DDMC branches in; the gray FP64 transport
// without DDMC runs the lean instantiation, which needs fewer registers.
//
// V = 2 is the convex-polyhedral form: the face search of
// distanceToNearestFace over the cell's inward normals and face centroids as
// written (alpha = ((faceCM - x).n) / (n.v), the first smallest positive).
template <int V, class RNG, class TALLY>
__device__ inline PhysOut physics_step(const Ctx &C, Track &T, RNG &rng, TALLY &tal) {
    // V: 0 gray Cartesian, 1 + multigroup and DDMC, 2 polyhedral, 3 = 1 + moving material,
    // 4 = 1 without the DDMC branch, 5 = 2 with DDMC (the variants without a
    // branch are smaller kernels for the instruction cache)
    constexpr bool FULL = V == 1 || V == 3 || V == 4, POLY = V == 2 || V == 5, HYDRO = V == 3,
                   DDMC = V == 1 || V == 3 || V == 5;
    PartReg &p = T.p;
    PhysOut o;
    o.status = NO_CELL_MOVE;
    o.face = -1;
    o.next = OUTSIDE;
    o.ghost = 0;
    o.usedRW = 0;
    o.errCode = 0;
    const uint32_t cell = p.cell;
    const uint32_t i = T.i, j = T.j, k = T.k;
    const double thr = EPSILON_FACE * T.speed;
    int face = -1;
    uint32_t next;
    double tFace;
    if constexpr (POLY) {
        const uint32_t k0 = C.cfo[cell], k1 = C.cfo[cell + 1];
        double minAlpha = DBL_MAX;
#pragma unroll 4
        for (uint32_t q = k0; q < k1; ++q) {
            const double4 n = C.cfN[q];
            const double nv = n.x * p.vx + n.y * p.vy + n.z * p.vz;
            if (nv >= -thr) continue;
            const double4 f = C.cfP[q];
            const double alpha = ((f.x - p.x) * n.x + (f.y - p.y) * n.y + (f.z - p.z) * n.z) / nv;
            if (alpha < minAlpha && alpha > 0) {
                minAlpha = alpha;
                face = static_cast<int>(q - k0);
            }
        }
        if (face < 0) { o.errCode = STORM_DERR_NO_FACE; return o; }
        tFace = minAlpha;
        const uint32_t nb = C.cfNext[k0 + face];
        next = nb < C.ncells ? nb : OUTSIDE;
        if (next == OUTSIDE) o.ghost = nb;
    }
    const double xl = POLY ? 0.0 : C.xe[i], xh = POLY ? 0.0 : C.xe[i + 1], yl = POLY ? 0.0 : C.ye[j],
                 yh = POLY ? 0.0 : C.ye[j + 1], zl = POLY ? 0.0 : C.ze[k], zh = POLY ? 0.0 : C.ze[k + 1];
    if constexpr (!POLY) {
    // candidate face per axis: numerator (p_f - x) and velocity component
    double nb = 0.0, vb = 1.0;
    {
        double n;
        bool ok;
        if (p.vx < -thr) { n = xl - p.x; ok = n < 0.0; } else if (p.vx > thr) { n = xh - p.x; ok = n > 0.0; } else ok = false;
        if (ok) { nb = n; vb = p.vx; face = p.vx > 0.0 ? 1 : 0; }
        if (p.vy < -thr) { n = yl - p.y; ok = n < 0.0; } else if (p.vy > thr) { n = yh - p.y; ok = n > 0.0; } else ok = false;
        if (ok && (face < 0 || fabs(n) * fabs(vb) < fabs(nb) * fabs(p.vy))) { nb = n; vb = p.vy; face = p.vy > 0.0 ? 3 : 2; }
        if (p.vz < -thr) { n = zl - p.z; ok = n < 0.0; } else if (p.vz > thr) { n = zh - p.z; ok = n > 0.0; } else ok = false;
        if (ok && (face < 0 || fabs(n) * fabs(vb) < fabs(nb) * fabs(p.vz))) { nb = n; vb = p.vz; face = p.vz > 0.0 ? 5 : 4; }
    }
    if (face < 0) { o.errCode = STORM_DERR_NO_FACE; return o; }
    tFace = nb / vb;
    if (!(tFace > 0.0)) { o.errCode = STORM_DERR_NO_FACE; return o; }
    switch (face) {
    case 0: next = (i > 0) ? cell - 1 : OUTSIDE; break;
    case 1: next = (i + 1 < C.nx) ? cell + 1 : OUTSIDE; break;
    case 2: next = (j > 0) ? cell - C.nx : OUTSIDE; break;
    case 3: next = (j + 1 < C.ny) ? cell + C.nx : OUTSIDE; break;
    case 4: next = (k > 0) ? cell - C.nx * C.ny : OUTSIDE; break;
    default: next = (k + 1 < C.nz) ? cell + C.nx * C.ny : OUTSIDE; break;
    }
    }
    double4 cp = C.phys[cell];
    double elastic = 0.0, eventOpacity = 0.0;
    // moving material: the lab-to-comoving Doppler factor (:1713-1720)
    double dop = 1.0;
    double4 cvel = make_double4(0.0, 0.0, 0.0, 1.0);
    if (HYDRO && C.withHydro) {
        cvel = C.vel[cell];
        dop = doppler_shift(C, cvel, p.vx, p.vy, p.vz);
    }
    if (FULL && C.groups >= 2) {
        // CalcAbsorptionOpacity at the particle's (comoving) frequency (:1742-1754)
        const double f = C.fleck[cell];
        const double absorptionOpacity = mg_absorption(C, cell, mg_clamp(C, HYDRO ? p.nu * dop : p.nu));
        elastic = C.sigS[cell];
        const double effectiveAbsorptionOpacity = (1.0 - f) * absorptionOpacity;
        eventOpacity = elastic + effectiveAbsorptionOpacity;
        cp.x = (eventOpacity > 0.0) ? 1.0 / eventOpacity : CUDART_INF;
        cp.y = absorptionOpacity * f * C.clight;
        cp.z = -1.0 / cp.y;
    }

    if (C.withRW && C.rwElig[cell]) {
        int r;
        if constexpr (POLY) {
            const PolyGeom g{&C, C.cfo[cell], C.cfo[cell + 1], C.mpx[cell], C.mpy[cell], C.mpz[cell]};
            r = try_random_walk<FULL>(C, p, rng, tal, cp, g);
        } else {
            const CartGeom g{xl, xh, yl, yh, zl, zh, C.xc[i], C.yc[j], C.zc[k]};
            r = try_random_walk<FULL, CartGeom, RNG, TALLY, HYDRO>(C, p, rng, tal, cp, g);
        }
        if (r == -2) { o.errCode = STORM_DERR_RW_SHRINK; return o; }
        if (r >= 0) {
            o.status = r;
            o.usedRW = 1;
            T.speed = vnorm(p.vx, p.vy, p.vz);
            return o;
        }
    }
    if (DDMC && (FULL || POLY) && C.withDDMC) {
        int dface = -1;
        uint32_t dnext = OUTSIDE;
        int r;
        if constexpr (POLY) {
            const PolyGeom g{&C, C.cfo[cell], C.cfo[cell + 1], C.mpx[cell], C.mpy[cell], C.mpz[cell]};
            r = try_ddmc_poly(C, p, rng, tal, g, dnext);
        } else {
            r = try_ddmc(C, p, rng, tal, xl, xh, yl, yh, zl, zh, dface, dnext);
        }
        if (r >= 0) {
            o.status = r;
            o.usedRW = 2;
            if (r == CELL_MOVE) {
                o.face = dface;
                o.next = dnext;
                T.speed = vnorm(p.vx, p.vy, p.vz);
            }
            return o;
        }
    }

    const double c = C.clight;
    const double lp = -log1p(rng.open() - 1.0);
    const double scatteringDistance = HYDRO ? cp.x * lp / dop : cp.x * lp;
    const double timeScattering = isfinite(scatteringDistance) ? scatteringDistance / T.speed : CUDART_INF;
    // std::min_element over {face, scatter, census}: first smallest wins
    int best = 0;
    double dt = tFace;
    if (timeScattering < dt) { best = 1; dt = timeScattering; }
    if (p.t < dt) { best = 2; dt = p.t; }
    p.t -= dt;
    const double tmp2 = cp.y;
    const double tmp = -dt * tmp2;
    // moving material: the weight and the momentum attenuate at the comoving
    // rate (expFactor1), the material and the tallies at the lab rate (expFactor2)
    const double e2 = expm1(tmp);
    const double e1 = HYDRO ? expm1(tmp * dop) : e2;
    double integrated = p.w * dt;
    if (fabs(tmp2 * dt) >= 1e-12) integrated = p.w * e2 * cp.z;
    p.x += p.vx * dt;
    p.y += p.vy * dt;
    p.z += p.vz * dt;
    if (!C.noFeedback) tal.mat(cell, -e2 * p.w);
    if (HYDRO && C.withHydro && !C.noFeedback) {   // (:1793-1798)
        const double a = -e1 * p.w;
        tal.mom(C, cell, a * p.vx * C.invC2, a * p.vy * C.invC2, a * p.vz * C.invC2);
    }
    tal.rad(cell, integrated);
    if constexpr (TALLY::kEg) tal.eg(C, cell, integrated, p.nu);
    p.w *= 1.0 + e1;
    if (fabs(p.w) < p.w0 * 1e-3) {
        if (!C.noFeedback) tal.mat(cell, p.w);
        o.status = REMOVE;
        return o;
    }
    if (best == 0) {
        o.status = CELL_MOVE;
        o.face = face;
        o.next = next;
        if (!POLY && next == OUTSIDE) o.ghost = C.ncells + face_index(C, i, j, k, face);
    } else if (best == 1) {
        const double oldVx = p.vx, oldVy = p.vy, oldVz = p.vz;
        if (FULL && C.groups >= 2) {
            // elastic or effective scatter (:1826-1852): both re-scatter
            // isotropically; an effective scatter re-emits from the spectrum
            const double eventRandom = rng.open() * eventOpacity;
            const bool effective = !(eventRandom < elastic);
            isotropic(rng, c, p.vx, p.vy, p.vz);
            p.nu = mg_clamp(C, HYDRO ? p.nu * dop : p.nu);
            if (effective) {
                p.nu = mg_thermal_energy(C, cell, rng.open());
                if (p.nu < 0.0) { o.errCode = STORM_DERR_MG_SAMPLE; return o; }
            }
        } else {
            rng.skip();   // event-type draw; both branches re-scatter isotropically
            isotropic(rng, c, p.vx, p.vy, p.vz);
        }
        if (HYDRO && C.withHydro) {   // the comoving scatter back to the lab frame (:1853-1871)
            const double weightBefore = p.w;
            p.w *= dop;
            lorentz_to_lab(C, cvel, p);
            if (C.groups >= 2) p.nu = mg_clamp(C, p.nu);
            if (!C.noFeedback) momentum_exchange(C, tal, cell, weightBefore, oldVx, oldVy, oldVz, p);
        }
        T.speed = vnorm(p.vx, p.vy, p.vz);
        o.status = NO_CELL_MOVE;
    } else {
        o.status = DONE;
    }
    return o;
}

// ------------------------------------------------------------------ FP32-tracking form
// A particle in the FP32-tracking form: cell index plus its offset from the cell
// centre and its direction in FP32; time, weight and initial weight in FP64.
struct Track32 {
    float qx, qy, qz, ux, uy, uz;
    double t, w, w0;
    uint32_t cell, i, j, k;
    // the constants of cell `cc`, kept in registers while the particle stays in it
    uint32_t cc;
    float4 cp;
    float hx, hy, hz;
    // multigroup: photon energy, and the cell's kT and sigma0 (cached with cp)
    float nu, kT, s0;
};

__device__ __forceinline__ float clampf(float v, float h) { return fminf(fmaxf(v, -h), h); }

// RandomWalk::sampleLeakTime / sampleRadius (radiation/RandomWalk.hpp:81-137)
// on the FP32 copies of the tables: the same binary search and interpolations.
__device__ inline float rw_sample_leak32(const RwTables &T, float xi) {
    const float target = 1.0f - xi;
    if (target >= T.surv32[0]) return __expf(T.logTau32[0]);
    if (target <= T.surv32[RW_TABLE - 1]) return __expf(T.logTau32[RW_TABLE - 1]);
    const int b = min(static_cast<int>(target * static_cast<float>(RW_LEAK_BUCKETS)), RW_LEAK_BUCKETS - 1);
    uint32_t first = T.leakStart32[b];
    while (first < RW_TABLE && T.surv32[first] > target) ++first;
    if (first == 0) return __expf(T.logTau32[0]);
    if (first == RW_TABLE) return __expf(T.logTau32[RW_TABLE - 1]);
    const float S0 = T.surv32[first - 1], S1 = T.surv32[first];
    const float frac = (S0 - target) / (S0 - S1);
    const float l0 = T.logTau32[first - 1], l1 = T.logTau32[first];
    return __expf(l0 + frac * (l1 - l0));
}

__device__ inline float rw_sample_radius32(const RwTables &T, float tau, float xi) {
    const float logTau = __logf(fminf(fmaxf(tau, 1e-8f), 64.0f));
    const float lmin = static_cast<float>(T.logMin), lmax = static_cast<float>(T.logMax);
    const float tauPos = (logTau - lmin) / (lmax - lmin) * static_cast<float>(RW_TABLE - 1);
    uint32_t tauIdx = static_cast<uint32_t>(fmaxf(tauPos, 0.0f));
    if (tauIdx > RW_TABLE - 2) tauIdx = RW_TABLE - 2;
    const float tauFrac = tauPos - static_cast<float>(tauIdx);
    const float xiPos = fminf(fmaxf(xi, 0.0f), 1.0f) * static_cast<float>(RW_RADIUS - 1);
    uint32_t xiIdx = static_cast<uint32_t>(xiPos);
    if (xiIdx > RW_RADIUS - 2) xiIdx = RW_RADIUS - 2;
    const float xiFrac = xiPos - static_cast<float>(xiIdx);
    const float *r0p = T.radius32 + static_cast<size_t>(tauIdx) * RW_RADIUS + xiIdx;
    const float *r1p = r0p + RW_RADIUS;
    const float r0 = r0p[0] + xiFrac * (r0p[1] - r0p[0]);
    const float r1 = r1p[0] + xiFrac * (r1p[1] - r1p[0]);
    return fminf(fmaxf(r0 + tauFrac * (r1 - r0), 0.0f), 1.0f);
}

// RadiationIMC::tryRandomWalkStep (radiation/RadiationIMC.hpp:1065-1276), gray, in
// the FP32-tracking form: cell-local FP32 geometry, FP64 time, weight and
// tallies, the same draws in the same order as the FP64 form.  Ro is the
// distance to the nearest face (the caller has checked Ro >= rwMinParticle /
// sigma_T); the diffusion coefficient c / (3 sigma_T) is cp.z * C.rwDiffPerReach.
// distance of local point (x, y, z) from face slot k's plane, inward positive
__device__ __forceinline__ float poly_dist32(const Ctx &C, uint32_t k, float x, float y, float z) {
    const float4 pl = C.cfN32[k];
    return pl.w + (x * pl.x + y * pl.y + z * pl.z);
}
template <bool POLY>
__device__ __forceinline__ bool inside32(const Ctx &C, uint32_t cell, float x, float y, float z, float hx, float hy,
                                         float hz) {
    if constexpr (POLY) {
        for (uint32_t k = C.cfo[cell]; k < C.cfo[cell + 1]; ++k)
            if (poly_dist32(C, k, x, y, z) < 0.0f) return false;
        return true;
    } else {
        return !(fabsf(x) > hx || fabsf(y) > hy || fabsf(z) > hz);
    }
}

template <bool MG, bool POLY = false, class RNG, class TALLY>
__device__ inline int rw_jump32(const Ctx &C, Track32 &T, RNG &rng, TALLY &tal, const float4 &cp, float Ro, float hx,
                                float hy, float hz, int &err) {
    const uint32_t cell = T.cell;
    // gray: D = c / (3 sigma_T) from the reach; multigroup: the PGRW cell data
    float D, sigAf;
    double fl = 0.0, sigmaA = 0.0, gammaRw = 1.0;
    if (MG) {
        const double4 g4 = C.pgrw[cell];
        D = cp.w;
        fl = cp.y;
        sigmaA = g4.y;
        gammaRw = g4.w;
        sigAf = static_cast<float>(sigmaA * fl);
    } else {
        D = cp.z * C.rwDiffPerReach;
        sigAf = cp.y;
    }
    const float tauLeak = rw_sample_leak32(C.rw, rng.rawf());
    const double tLeak = static_cast<double>(tauLeak * (Ro * Ro) / D);
    double tUp = DBL_MAX;
    if (MG && gammaRw < 1.0 && sigmaA > 0.0 && fl > 0.0) {   // PGRW upscatter (radiation/RadiationIMC.hpp:1130-1135)
        const float xiUp = rng.rawf();
        tUp = -static_cast<double>(__logf(xiUp)) / (C.clight * (1.0 - fl) * sigmaA * (1.0 - gammaRw));
    }
    int ev;
    double dt;
    if (tLeak <= T.t && tLeak <= tUp) { ev = 0; dt = tLeak; }
    else if (T.t <= tUp) { ev = 1; dt = T.t; }
    else { ev = 2; dt = tUp; }
    const float tau = sigAf * static_cast<float>(dt * C.clight);
    const double e1 = static_cast<double>(expm1f(-tau));
    if (!C.noFeedback) tal.mat(cell, -e1 * T.w);
    if (sigAf > 0.0f) {
        const double invRate = MG ? -1.0 / (static_cast<double>(sigAf) * C.clight) : static_cast<double>(cp.w);
        tal.rad(cell, T.w * e1 * invRate);
        if constexpr (TALLY::kEg) tal.eg32(C, cell, T.w * e1 * invRate, T.nu);
    }
    T.w *= 1.0 + e1;
    T.t -= dt;
    if (fabs(T.w) < T.w0 * 1e-4) {
        if (!C.noFeedback) tal.mat(cell, T.w);
        return OUT_CUTOFF;
    }
    const float cosT = 2.0f * rng.rawf() - 1.0f;
    const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
    float sphi, cphi;
    __sincosf(6.2831853f * rng.rawf(), &sphi, &cphi);
    const float dx = sinT * cphi, dy = sinT * sphi, dz = cosT;
    float disp = Ro;
    if (ev != 0) {
        const float tauPos = static_cast<float>(dt) * D / (Ro * Ro);
        disp = fminf(Ro * rw_sample_radius32(C.rw, tauPos, rng.rawf()), Ro);
    }
    const float nudge = 1.0f - static_cast<float>(RW_NUDGE);   // toward the cell centre (local origin)
    float lx = (T.qx + disp * dx) * nudge, ly = (T.qy + disp * dy) * nudge, lz = (T.qz + disp * dz) * nudge;
    int guard = 0;
    while (!inside32<POLY>(C, cell, lx, ly, lz, hx, hy, hz)) {
        disp *= 0.99f;
        lx = T.qx + disp * dx;
        ly = T.qy + disp * dy;
        lz = T.qz + disp * dz;
        if (++guard > RW_SHRINK_CAP) { err = STORM_DERR_RW_SHRINK; return OUT_ERROR; }
    }
    T.qx = lx; T.qy = ly; T.qz = lz;
    const float theta = 6.2831853f * rng.rawf();
    const float cz = 2.0f * rng.rawf() - 1.0f;
    const float sz = sqrtf(fmaxf(0.0f, 1.0f - cz * cz));
    float st, ct;
    __sincosf(theta, &st, &ct);
    T.ux = sz * ct; T.uy = sz * st; T.uz = cz;
    if (MG && ev == 2) {   // upscatter: a frequency above the cutoff (:1232-1250)
        const uint32_t cutoff = C.pgrwCut[cell];
        const double *cdf = C.mgCdf + static_cast<size_t>(cell) * (C.groups + 1);
        const double cdfAtCutoff = cdf[cutoff], cdfTotal = cdf[C.groups];
        if (cdfTotal > cdfAtCutoff)   // sampled at the start of the next segment (segment32)
            T.nu = -1.0f - static_cast<float>(cdfAtCutoff / cdfTotal);
        else
            T.nu = static_cast<float>(mg_clamp(C, nextafter(C.gb[cutoff], DBL_MAX)));
    }
    return ev == 1 ? OUT_CENSUS : OUT_CONTINUE;
}

// tryDDMCStep (radiation/RadiationIMC.hpp:1416-1612) in the FP32-tracking form:
// the event time from the cell's total leak rate, attenuation at sigma_A f c
// with FP64 weight, time and tallies, then census, cutoff or a leak through a
// face picked by the cumulative face fractions.  A leaking particle enters
// the neighbour at the centre of the shared face (ENTRY32 inside it) with a
// cosine-law direction about the face normal.  The caller has checked the
// particle's distance to the faces against the cell's DDMC depth.
template <class RNG, class TALLY>
__device__ inline int ddmc_jump32(const Ctx &C, Track32 &T, RNG &rng, TALLY &tal, const float4 &da) {
    const uint32_t cell = T.cell;
    const double tEvent = static_cast<double>(-__logf(rng.rawf()) * da.y);
    const bool census = T.t <= tEvent;
    const double dt = census ? T.t : tEvent;
    const float tau = da.z * static_cast<float>(dt);
    const double e1 = static_cast<double>(expm1f(-tau));
    if (!C.noFeedback) tal.mat(cell, -e1 * T.w);
    tal.rad(cell, da.z > 0.0f ? T.w * e1 * (-1.0 / static_cast<double>(da.z)) : T.w * dt);
    if constexpr (TALLY::kEg)
        tal.eg32(C, cell, da.z > 0.0f ? T.w * e1 * (-1.0 / static_cast<double>(da.z)) : T.w * dt, T.nu);
    T.w *= 1.0 + e1;
    T.t -= dt;
    if (fabs(T.w) < T.w0 * 1e-3) {
        if (!C.noFeedback) tal.mat(cell, T.w);
        return OUT_CUTOFF;
    }
    if (census) return OUT_CENSUS;
    const float4 c0 = C.ddmc32[3 * static_cast<size_t>(cell) + 1], c1 = C.ddmc32[3 * static_cast<size_t>(cell) + 2];
    const float u = rng.rawf();
    int s = static_cast<int>(c1.z);   // the last face with a leak rate
    if (u <= c0.x) s = 0;
    else if (u <= c0.y) s = 1;
    else if (u <= c0.z) s = 2;
    else if (u <= c0.w) s = 3;
    else if (u <= c1.x) s = 4;
    else if (u <= c1.y) s = 5;
    if (s < 0) return OUT_CENSUS;
    const float mu = sqrtf(rng.rawf());
    const float phi = 6.2831853f * rng.rawf();
    const float st = sqrtf(fmaxf(0.0f, 1.0f - mu * mu));
    float sp, cph;
    __sincosf(phi, &sp, &cph);
    const float sg = (s & 1) ? 1.0f : -1.0f;
    switch (s) {
    case 0: --T.i; T.cell -= 1; T.qx = C.hx[T.i] * ENTRY32; break;
    case 1: ++T.i; T.cell += 1; T.qx = -C.hx[T.i] * ENTRY32; break;
    case 2: --T.j; T.cell -= C.nx; T.qy = C.hy[T.j] * ENTRY32; break;
    case 3: ++T.j; T.cell += C.nx; T.qy = -C.hy[T.j] * ENTRY32; break;
    case 4: --T.k; T.cell -= C.nx * C.ny; T.qz = C.hz[T.k] * ENTRY32; break;
    default: ++T.k; T.cell += C.nx * C.ny; T.qz = -C.hz[T.k] * ENTRY32; break;
    }
    const int axis = s >> 1;
    if (axis == 0) { T.qy = 0.0f; T.qz = 0.0f; T.ux = sg * mu; T.uy = st * cph; T.uz = st * sp; }
    else if (axis == 1) { T.qz = 0.0f; T.qx = 0.0f; T.uy = sg * mu; T.uz = st * cph; T.ux = st * sp; }
    else { T.qx = 0.0f; T.qy = 0.0f; T.uz = sg * mu; T.ux = st * cph; T.uy = st * sp; }
    return OUT_CONTINUE;
}

// tryDDMCStep in the FP32-tracking form on a convex-polyhedral cell: the
// same event, attenuation and tallies as ddmc_jump32; the leak face is picked
// by the per-slot cumulative fractions, and the particle enters the neighbour
// at the face centroid (offset from the neighbour's mesh point, nudged
// ENTRY32 toward it) with a cosine-law direction about the face's unit normal
// turned toward the neighbour.
template <class RNG, class TALLY>
__device__ inline int ddmc_jump32_poly(const Ctx &C, Track32 &T, RNG &rng, TALLY &tal, const float4 &da) {
    const uint32_t cell = T.cell;
    const double tEvent = static_cast<double>(-__logf(rng.rawf()) * da.y);
    const bool census = T.t <= tEvent;
    const double dt = census ? T.t : tEvent;
    const float tau = da.z * static_cast<float>(dt);
    const double e1 = static_cast<double>(expm1f(-tau));
    if (!C.noFeedback) tal.mat(cell, -e1 * T.w);
    tal.rad(cell, da.z > 0.0f ? T.w * e1 * (-1.0 / static_cast<double>(da.z)) : T.w * dt);
    T.w *= 1.0 + e1;
    T.t -= dt;
    if (fabs(T.w) < T.w0 * 1e-3) {
        if (!C.noFeedback) tal.mat(cell, T.w);
        return OUT_CUTOFF;
    }
    if (census) return OUT_CENSUS;
    const uint32_t k0 = C.cfo[cell], k1 = C.cfo[cell + 1];
    const float u = rng.rawf();
    int last = static_cast<int>(C.ddmc32[3 * static_cast<size_t>(cell) + 2].z);   // the last slot with a leak rate
    if (last < 0) return OUT_CENSUS;
    uint32_t k = k0 + static_cast<uint32_t>(last);
    for (uint32_t q = k0; q < k1; ++q)
        if (u <= C.ddmcCum32[q]) { k = q; break; }
    const uint32_t nb = C.cfNext[k];
    const float4 pl = C.cfN32[k];
    float n0 = -pl.x, n1 = -pl.y, n2 = -pl.z;   // outward: toward the neighbour
    const float tx = static_cast<float>(C.mpx[nb] - C.mpx[cell]), ty = static_cast<float>(C.mpy[nb] - C.mpy[cell]),
                tz = static_cast<float>(C.mpz[nb] - C.mpz[cell]);
    if (n0 * tx + n1 * ty + n2 * tz < 0.0f) { n0 = -n0; n1 = -n1; n2 = -n2; }
    const float mu = sqrtf(rng.rawf());
    const float phi = 6.2831853f * rng.rawf();
    const float st = sqrtf(fmaxf(0.0f, 1.0f - mu * mu));
    float sp, cph;
    __sincosf(phi, &sp, &cph);
    float h0 = 0.0f, h1 = 0.0f;
    if (fabsf(n0) < 0.9f) h0 = 1.0f; else h1 = 1.0f;
    const float hn = h0 * n0 + h1 * n1;
    float a0 = h0 - n0 * hn, a1 = h1 - n1 * hn, a2 = -n2 * hn;
    const float am = rsqrtf(fmaxf(a0 * a0 + a1 * a1 + a2 * a2, 1e-30f));
    a0 *= am; a1 *= am; a2 *= am;
    const float b0 = n1 * a2 - n2 * a1, b1 = n2 * a0 - n0 * a2, b2 = n0 * a1 - n1 * a0;
    float dx = mu * n0 + st * (cph * a0 + sp * b0);
    float dy = mu * n1 + st * (cph * a1 + sp * b1);
    float dz = mu * n2 + st * (cph * a2 + sp * b2);
    const float dm = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-30f));
    T.ux = dx * dm; T.uy = dy * dm; T.uz = dz * dm;
    const double4 fcm = C.cfP[k];
    T.qx = static_cast<float>(fcm.x - C.mpx[nb]) * ENTRY32;
    T.qy = static_cast<float>(fcm.y - C.mpy[nb]) * ENTRY32;
    T.qz = static_cast<float>(fcm.z - C.mpz[nb]) * ENTRY32;
    T.cell = nb;
    T.i = nb;
    return OUT_CONTINUE;
}

// findGroup on the FP32 form's float bounds (the same rule)
__device__ __forceinline__ void SegmentTallyEg::eg32(const Ctx &C, uint32_t c, double v, float nu) {
    uint32_t lo = 0, hi = C.groups - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (nu < C.gb32[mid + 1]) hi = mid; else lo = mid + 1;
    }
    atomicAdd(C.egAvg + static_cast<size_t>(c) * C.groups + lo, v);
}

// Multigroup absorption opacity in FP32 from the cell's cached kT and
// sigma0 / (kT)^q: at the group centre E_g^p comes from the per-group table.
__device__ __forceinline__ float mg_absorption32(const Ctx &C, const Track32 &T, float nu) {
    float E, v;
    if (C.mgGroupConst) {
        uint32_t lo = 0, hi = C.groups - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (nu < C.gb32[mid + 1]) hi = mid; else lo = mid + 1;
        }
        E = C.gc32[lo];
        v = T.s0 / C.mgEp32[lo];
    } else {
        E = fmaxf(nu, C.gb32[0]);
        v = T.s0 / __powf(E, static_cast<float>(C.mgP));
    }
    if (C.mgS != 0.0) {
        const float x = -expm1f(-E / T.kT);
        v *= (C.mgS == 1.0) ? x : __powf(x, static_cast<float>(C.mgS));
    }
    return v;
}

// One segment plus the manager's handling, in the FP32-tracking form.  Same
// events, same draws per event and the same FP64 tally updates as the FP64
// form; distances, the face search and the collision distance are FP32 in the
// cell's own frame, so precision follows the cell size, not the domain.
//
// Face search: along each axis the exit plane is n_a = h_a - sign(u_a) q_a away
// at speed |u_a|; the nearest exit is found by cross-multiplied comparisons
// (n_a |u_b| < n_b |u_a|, first smallest wins, an axis with u_a = 0 never
// wins) and only the winner is divided.
//
// POLY: a convex-polyhedral cell; the offset is from the cell's mesh point and
// each face is the plane n.q + h = 0 (n inward, h the mesh point's distance).
// The exit is the first smallest (n.q + h) / (-n.u) over faces the direction
// approaches; a particle that changes cells re-expresses its offset from the
// new mesh point and is nudged 2^-21 of it toward that point.
// DDMC = false compiles the DDMC branch out (problems without withDDMC): a
// smaller kernel for the instruction cache.
template <bool MG, class RNG, class TALLY, bool POLY = false, bool DDMC = true>
__device__ inline int segment32(const Ctx &C, Track32 &T, RNG &rng, TALLY &tal, int &usedRW, int &err) {
    const uint32_t cell = T.cell;
    if (T.cc != cell) {   // entered another cell: load its constants once
        T.cp = C.phys32[cell];
        if (!POLY) { T.hx = C.hx[T.i]; T.hy = C.hy[T.j]; T.hz = C.hz[T.k]; }
        T.cc = cell;
        if (MG) {
            T.kT = static_cast<float>(mg_kT(C, cell));
            T.s0 = static_cast<float>(C.sig0[cell] / C.mgKTq[cell]);   // sigma0 / (kT)^q
        }
    }
    const float hx = T.hx, hy = T.hy, hz = T.hz;
    const float4 cp = T.cp;
    if (MG) {
        // A re-emission from the cell's spectrum that the previous segment
        // (an effective scatter, or a PGRW upscatter that draws above the
        // cutoff's cumulative fraction lo) left pending as nu = -(1 + lo): it
        // is sampled here, so that the kernel holds one copy of the sampler.
        if (T.nu < 0.0f) {
            const double lo = static_cast<double>(-T.nu - 1.0f);
            const double nu = mg_thermal_energy(C, cell, lo + static_cast<double>(rng.rawf()) * (1.0 - lo));
            if (nu < 0.0) { err = STORM_DERR_MG_SAMPLE; return OUT_ERROR; }
            T.nu = static_cast<float>(nu);
        }
        T.nu = fminf(fmaxf(T.nu, C.gb32[0]), C.gb32[C.groups]);   // clampFrequencyToBounds
    }

    // Random Walk only where the particle is at least cp.z = rwMinParticleOpticalDepth / sigma_T
    // from every face (cp.z is inf in cells that are not eligible); in a multigroup
    // problem only below the cell's PGRW group cutoff
    float Ro;
    if constexpr (POLY) {
        // only Random Walk and DDMC cells (finite reach) need the distance to the faces
        Ro = 0.0f;
        const bool ddmcCell = DDMC && C.withDDMC && C.ddmc32[3 * static_cast<size_t>(cell)].x < CUDART_INF_F;
        if (cp.z < CUDART_INF_F || ddmcCell) {
            Ro = FLT_MAX;
#pragma unroll 4
            for (uint32_t k = C.cfo[cell]; k < C.cfo[cell + 1]; ++k) Ro = fminf(Ro, poly_dist32(C, k, T.qx, T.qy, T.qz));
        }
    } else {
        Ro = fminf(fminf(hx - fabsf(T.qx), hy - fabsf(T.qy)), hz - fabsf(T.qz));
    }
    if (Ro >= cp.z && Ro > 0.0f && (!MG || static_cast<double>(T.nu) < C.gb[C.pgrwCut[cell]])) {
        usedRW = 1;
        return rw_jump32<MG, POLY>(C, T, rng, tal, cp, Ro, hx, hy, hz, err);
    }
    if (DDMC && C.withDDMC) {   // DDMC after a Random Walk that was not taken (:1723-1738)
        const float4 da = C.ddmc32[3 * static_cast<size_t>(cell)];   // depth reach, 1/total, sigma_A f c, nu bound
        if (Ro >= da.x && Ro > 0.0f && (!MG || T.nu < da.w)) {
            if constexpr (POLY) return ddmc_jump32_poly(C, T, rng, tal, da);
            else return ddmc_jump32(C, T, rng, tal, da);
        }
    }
    // gray: the cell constants; multigroup: the opacity at the particle's frequency
    float invSigE, sigAf, sigE = 0.0f, elastic = 0.0f;
    double invRate;
    if (MG) {
        const float sigA = mg_absorption32(C, T, T.nu);
        const float f = cp.y;
        elastic = cp.x;
        sigE = elastic + (1.0f - f) * sigA;
        invSigE = sigE > 0.0f ? 1.0f / sigE : CUDART_INF_F;
        sigAf = sigA * f;
        invRate = -1.0 / (static_cast<double>(sigAf) * C.clight);
    } else {
        invSigE = cp.x;
        sigAf = cp.y;
        invRate = static_cast<double>(cp.w);
    }

    int face = -1;
    float sF;
    if constexpr (POLY) {
        float bestS = FLT_MAX;
        const uint32_t k0 = C.cfo[cell], k1 = C.cfo[cell + 1];
#pragma unroll 4
        for (uint32_t k = k0; k < k1; ++k) {
            const float4 pl = C.cfN32[k];
            const float un = T.ux * pl.x + T.uy * pl.y + T.uz * pl.z;
            if (un >= 0.0f) continue;
            const float d = fmaxf(pl.w + (T.qx * pl.x + T.qy * pl.y + T.qz * pl.z), 0.0f);
            const float sk = d / -un;
            if (sk < bestS) { bestS = sk; face = static_cast<int>(k - k0); }
        }
        if (face < 0) { err = STORM_DERR_NO_FACE; return OUT_ERROR; }
        sF = bestS;
    } else {
    const float ax = fabsf(T.ux), ay = fabsf(T.uy), az = fabsf(T.uz);
    const float nxp = ax > 0.0f ? fmaxf(hx - (T.ux > 0.0f ? T.qx : -T.qx), 0.0f) : 1.0f;
    const float nyp = ay > 0.0f ? fmaxf(hy - (T.uy > 0.0f ? T.qy : -T.qy), 0.0f) : 1.0f;
    const float nzp = az > 0.0f ? fmaxf(hz - (T.uz > 0.0f ? T.qz : -T.qz), 0.0f) : 1.0f;
    float bn = nxp, bd = ax;
    face = ax > 0.0f ? (T.ux > 0.0f ? 1 : 0) : -1;
    if (ay > 0.0f && (face < 0 || nyp * bd < bn * ay)) { bn = nyp; bd = ay; face = T.uy > 0.0f ? 3 : 2; }
    if (az > 0.0f && (face < 0 || nzp * bd < bn * az)) { bn = nzp; bd = az; face = T.uz > 0.0f ? 5 : 4; }
    if (face < 0) { err = STORM_DERR_NO_FACE; return OUT_ERROR; }
    sF = __fdividef(bn, bd);
    }
    const double c = C.clight;

    const float sC = invSigE * (-__logf(rng.rawf()));
    const float sL = static_cast<float>(T.t * c);
    int best = 0;
    float ds = sF;
    if (sC < ds) { best = 1; ds = sC; }
    if (sL < ds) { best = 2; ds = sL; }
    const double dt = (best == 2) ? T.t : static_cast<double>(ds) * C.invC;
    T.t -= dt;
    const float tau = sigAf * ds;
    const double e1 = static_cast<double>(expm1f(-tau));
    double integrated = T.w * dt;
    if (tau >= 1e-12f) integrated = T.w * e1 * invRate;
    if constexpr (POLY) {
        T.qx = fmaf(T.ux, ds, T.qx);
        T.qy = fmaf(T.uy, ds, T.qy);
        T.qz = fmaf(T.uz, ds, T.qz);
    } else {
        T.qx = clampf(fmaf(T.ux, ds, T.qx), hx);
        T.qy = clampf(fmaf(T.uy, ds, T.qy), hy);
        T.qz = clampf(fmaf(T.uz, ds, T.qz), hz);
    }
    if (!C.noFeedback) tal.mat(cell, -e1 * T.w);
    tal.rad(cell, integrated);
    if constexpr (TALLY::kEg) tal.eg32(C, cell, integrated, T.nu);
    T.w *= 1.0 + e1;
    if (fabs(T.w) < T.w0 * 1e-3) {
        if (!C.noFeedback) tal.mat(cell, T.w);
        return OUT_CUTOFF;
    }
    if (best == 2) return OUT_CENSUS;
    if (best == 1) {
        bool effective = false;
        if (MG) effective = !(rng.rawf() * sigE < elastic);   // elastic or effective scatter
        else rng.skip();   // the event-type draw (a no-op on the FP32 form's own stream)
        const float theta = 6.2831853f * rng.rawf();
        const float cosT = 2.0f * rng.rawf() - 1.0f;
        const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
        float st, ct;
        __sincosf(theta, &st, &ct);
        T.ux = sinT * ct; T.uy = sinT * st; T.uz = cosT;
        if (MG && effective) T.nu = -1.0f;   // re-emission from the cell's spectrum, at the next segment's start
        return OUT_CONTINUE;
    }
    // face crossing
    if constexpr (POLY) {
        const uint32_t k = C.cfo[cell] + static_cast<uint32_t>(face);
        const uint32_t nb = C.cfNext[k];
        if (nb < C.ncells) {
            // the offset from the new cell's mesh point, nudged toward it
            const float dx = static_cast<float>(C.mpx[cell] - C.mpx[nb]);
            const float dy = static_cast<float>(C.mpy[cell] - C.mpy[nb]);
            const float dz = static_cast<float>(C.mpz[cell] - C.mpz[nb]);
            T.qx = (T.qx + dx) * ENTRY32;
            T.qy = (T.qy + dy) * ENTRY32;
            T.qz = (T.qz + dz) * ENTRY32;
            T.cell = nb;
            T.i = nb;
            return OUT_CONTINUE;
        }
        // a box face: its axis and side from the inward normal
        const float4 pl = C.cfN32[k];
        const float apx = fabsf(pl.x), apy = fabsf(pl.y), apz = fabsf(pl.z);
        const int ax = (apx >= apy && apx >= apz) ? 0 : (apy >= apz ? 1 : 2);
        const float na = ax == 0 ? pl.x : (ax == 1 ? pl.y : pl.z);
        const int bface = 2 * ax + (na < 0.0f ? 1 : 0);
        if (C.escapeNoCheck || C.bf[bface].action == STORM_FACE_ESCAPE) return OUT_ESCAPE;
        if (ax == 0) T.ux = -T.ux; else if (ax == 1) T.uy = -T.uy; else T.uz = -T.uz;
        // back inside by the reflection nudge, measured from the face plane
        const float d = pl.w + (T.qx * pl.x + T.qy * pl.y + T.qz * pl.z);
        const float push = C.reflNudge[bface] - d;
        T.qx += push * pl.x; T.qy += push * pl.y; T.qz += push * pl.z;
        return OUT_CONTINUE;
    }
    const int axis = face >> 1, hi = face & 1;
    bool inside;
    switch (face) {
    case 0: inside = T.i > 0; break;
    case 1: inside = T.i + 1 < C.nx; break;
    case 2: inside = T.j > 0; break;
    case 3: inside = T.j + 1 < C.ny; break;
    case 4: inside = T.k > 0; break;
    default: inside = T.k + 1 < C.nz; break;
    }
    if (inside) {
        // The serial manager nudges a particle that changed cells 1e-8 of the
        // way to the new cell's centre (MonteCarloManagerSerial.hpp:323-327),
        // which an FP32 offset cannot hold.  The particle enters ENTRY32 of
        // the half width from the centre instead: at least 4 ulps inside the
        // face, so a cell whose mean free path is below the offset's
        // resolution still sees a nonzero distance to the face (Random Walk
        // eligible) rather than a particle pinned to the face.
        switch (face) {
        case 0: --T.i; T.cell -= 1; T.qx = C.hx[T.i] * ENTRY32; break;
        case 1: ++T.i; T.cell += 1; T.qx = -C.hx[T.i] * ENTRY32; break;
        case 2: --T.j; T.cell -= C.nx; T.qy = C.hy[T.j] * ENTRY32; break;
        case 3: ++T.j; T.cell += C.nx; T.qy = -C.hy[T.j] * ENTRY32; break;
        case 4: --T.k; T.cell -= C.nx * C.ny; T.qz = C.hz[T.k] * ENTRY32; break;
        default: ++T.k; T.cell += C.nx * C.ny; T.qz = -C.hz[T.k] * ENTRY32; break;
        }
        return OUT_CONTINUE;
    }
    // the box face this cell face lies on (GetBoxFaces order matches the side order)
    if (C.escapeNoCheck || C.bf[face].action == STORM_FACE_ESCAPE) return OUT_ESCAPE;
    const float sgn = hi ? 1.0f : -1.0f;
    if (axis == 0) { T.ux = -T.ux; T.qx = sgn * (hx - fminf(C.reflNudge[face], 0.25f * hx)); }
    else if (axis == 1) { T.uy = -T.uy; T.qy = sgn * (hy - fminf(C.reflNudge[face], 0.25f * hy)); }
    else { T.uz = -T.uz; T.qz = sgn * (hz - fminf(C.reflNudge[face], 0.25f * hz)); }
    return OUT_CONTINUE;
}

// ------------------------------------------------------------------ boundary
// BoundaryCondition::getInwardBoxFaceNormalIfClose (:61-85) with host-precomputed face data.
__device__ __forceinline__ bool box_face_close(const BoxFaceDev &F, double x, double y, double z) {
    if (!F.valid) return false;
    double pd = F.raw[0] * (x - F.on[0]) + F.raw[1] * (y - F.on[1]) + F.raw[2] * (z - F.on[2]);
    return fabs(pd) < F.thresh;
}
// reflectParticleOnBoxFace (:87-108)
__device__ __forceinline__ void box_face_reflect(const BoxFaceDev &F, PartReg &p) {
    double sd = (p.x - F.on[0]) * F.unit[0] + (p.y - F.on[1]) * F.unit[1] + (p.z - F.on[2]) * F.unit[2];
    p.x -= sd * F.unit[0];
    p.y -= sd * F.unit[1];
    p.z -= sd * F.unit[2];
    p.x += F.nudge * F.unit[0];
    p.y += F.nudge * F.unit[1];
    p.z += F.nudge * F.unit[2];
    double vn = p.vx * F.unit[0] + p.vy * F.unit[1] + p.vz * F.unit[2];
    if (vn < 0.0) {
        double s2 = 2.0 * vn;
        p.vx -= s2 * F.unit[0];
        p.vy -= s2 * F.unit[1];
        p.vz -= s2 * F.unit[2];
    }
}

// The serial manager's handling of one RadiationIMC::step result
// (manager/MonteCarloManagerSerial.hpp:318-369), with BoundaryCondition::apply
// for the per-face descriptor (VacuumBoundary, RigidBoundary, SideTemperature,
// TwoSidesTemperature all lower to it).
template <bool POLY = false>
__device__ __forceinline__ int manager_handle(const Ctx &C, Track &T, const PhysOut &o) {
    PartReg &p = T.p;
    if (o.status == CELL_MOVE) {
        if (POLY && o.next != OUTSIDE) {
            const uint32_t nc = o.next;
            p.x = (1 - MONTECARLO_EPS) * p.x + MONTECARLO_EPS * C.mpx[nc];
            p.y = (1 - MONTECARLO_EPS) * p.y + MONTECARLO_EPS * C.mpy[nc];
            p.z = (1 - MONTECARLO_EPS) * p.z + MONTECARLO_EPS * C.mpz[nc];
            p.cell = nc;
            T.i = nc;
            return OUT_CONTINUE;
        }
        if (o.next != OUTSIDE) {
            switch (o.face) {
            case 0: --T.i; break;
            case 1: ++T.i; break;
            case 2: --T.j; break;
            case 3: ++T.j; break;
            case 4: --T.k; break;
            default: ++T.k; break;
            }
            p.x = (1 - MONTECARLO_EPS) * p.x + MONTECARLO_EPS * C.xc[T.i];
            p.y = (1 - MONTECARLO_EPS) * p.y + MONTECARLO_EPS * C.yc[T.j];
            p.z = (1 - MONTECARLO_EPS) * p.z + MONTECARLO_EPS * C.zc[T.k];
            p.cell = o.next;
            return OUT_CONTINUE;
        }
        if (C.escapeNoCheck) return OUT_ESCAPE;
        bool reflected = false;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if (box_face_close(C.bf[f], p.x, p.y, p.z)) {
                if (C.bf[f].action == STORM_FACE_ESCAPE) return OUT_ESCAPE;
                box_face_reflect(C.bf[f], p);
                reflected = true;
            }
        }
        if (!reflected) return OUT_ERROR;
        T.speed = vnorm(p.vx, p.vy, p.vz);
        const double mx = POLY ? C.mpx[p.cell] : C.xc[T.i], my = POLY ? C.mpy[p.cell] : C.yc[T.j],
                     mz = POLY ? C.mpz[p.cell] : C.zc[T.k];
        p.x = (1 - MONTECARLO_EPS) * p.x + MONTECARLO_EPS * mx;
        p.y = (1 - MONTECARLO_EPS) * p.y + MONTECARLO_EPS * my;
        p.z = (1 - MONTECARLO_EPS) * p.z + MONTECARLO_EPS * mz;
        return OUT_CONTINUE;
    }
    if (o.status == REMOVE) return OUT_CUTOFF;
    if (o.status == DONE) return OUT_CENSUS;
    return OUT_CONTINUE;
}

}  // namespace storm
