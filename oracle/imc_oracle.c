/*
 * Test infrastructure only -- the oracle.  Plain-C restatement of STORM's gray
 * IMC hot path, used by tests/ (and by __graft_entry__.smoke and bench.py's
 * CPU baseline leg) as the checker of the CUDA engine.  The product never
 * links, loads or calls this file.
 *
 * Every function below names the reference lines it restates.  Floating-point
 * expressions keep the reference's association and operand order (gcc at -O2
 * on x86-64 emits no FMA, like the reference build), so on a shared tape of
 * uniforms this code and the reference build agree bit for bit.
 *
 * Random numbers: a Rng is either a tape (replay of the reference's recorded
 * draws) or the engine's counter-based stream: Philox4x32-10 (Salmon, Moraes,
 * Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11) with
 *   key     = (low 32 bits of seed, high 32 bits of seed)
 *   counter = (draw >> 1, pid, step, tag)
 * and uniform = (m + 0.5) * 2^-52 from a 52-bit integer m built from words
 * (0,1) for even draws and (2,3) for odd draws.  Tags: 1 transport (pid =
 * particle index in the step's bank), 2 cell emission (pid = packet index),
 * 3 face emission, 4 comb (pid = cell).
 */
#include "imc_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { NO_CELL_MOVE = 0, CELL_MOVE = 1, DONE = 2, REMOVE = 3, REFLECT = 4 }; /* particle/ParticleStatus.hpp:8-15 */
enum { TAG_TRANSPORT = 1, TAG_CELL_EMIT = 2, TAG_FACE_EMIT = 3, TAG_COMB = 4 };

#define EPSILON_FACE 1e-12          /* particle/Particle.hpp:17 */
#define MONTECARLO_EPS 1e-8         /* manager/MonteCarloConfig.hpp:11 */
#define RW_NUDGE 1e-6               /* radiation/RadiationIMC.hpp:1211 */
#define REFLECT_NUDGE 1e-6          /* boundary/BoundaryCondition.hpp:100 */
#define HISTORY_SEGMENT_CAP 100000000ULL

/* ------------------------------------------------------------------ RNG */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static double u52(uint32_t a, uint32_t b) {
    uint64_t m = ((uint64_t)(a >> 6) << 26) | (uint64_t)(b >> 6);
    return ((double)m + 0.5) * 0x1p-52;
}

double orc_uniform(uint64_t seed, uint32_t tag, uint32_t step, uint32_t pid, uint32_t draw) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t ctr[4] = {draw >> 1, pid, step, tag};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    return (draw & 1u) ? u52(o[2], o[3]) : u52(o[0], o[1]);
}

/* MurmurHash3's 32-bit finaliser (a bijection on 32-bit words). */
static uint32_t fmix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
    return h;
}
/* Comb shuffle key: a keyed bijection of [0, 2^b) applied to the particle
 * index (every pid of the step is below 2^b), so sorting by (cell << b | key)
 * is a pseudo-random permutation within each cell with no ties.  Xor with the
 * step key, then odd multiplications and xor-shifts, each invertible mod 2^b. */
uint32_t orc_comb_key(uint64_t seed, uint32_t step, uint32_t pid, int b) {
    uint32_t k = fmix32((uint32_t)seed ^ fmix32(step * 0x9E3779B9u + (uint32_t)(seed >> 32)));
    const uint32_t mask = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
    uint32_t h = (pid ^ k) & mask;
    h = (h * 0x9E3779B1u) & mask;
    h ^= h >> ((b + 1) / 2);
    h = (h * 0x85EBCA77u) & mask;
    h ^= h >> ((b + 2) / 3);
    h = (h * 0xC2B2AE3Du) & mask;
    h ^= h >> ((b + 1) / 2);
    return h;
}
/* the comb key width: the smallest b >= 1 with 2^b >= pidLimit */
static int pid_bits(uint64_t pidLimit) {
    int b = 1;
    while (b < 32 && (1ull << b) < pidLimit) ++b;
    return b;
}

typedef struct {
    int tape_mode;
    const double *tape;
    uint32_t len, pos;
    int exhausted;
    uint64_t seed;
    uint32_t tag, step, pid, draw;
} Rng;

static double rng_raw(Rng *r) {
    if (r->tape_mode) {
        if (r->pos >= r->len) { r->exhausted = 1; return 0.5; }
        return r->tape[r->pos++];
    }
    return orc_uniform(r->seed, r->tag, r->step, r->pid, r->draw++);
}
/* RadiationIMC::randomUnitOpen (radiation/RadiationIMC.hpp:700-713) */
static double rng_open(Rng *r) {
    double v = rng_raw(r);
    if (v <= 0.0) return DBL_MIN;
    if (v >= 1.0) return nextafter(1.0, 0.0);
    return v;
}

/* ------------------------------------------------------------------ vectors (elementary/PointOps.hpp) */
typedef struct { double x, y, z; } V3;
static V3 v3(double x, double y, double z) { V3 r = {x, y, z}; return r; }
static V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static V3 vscale(double s, V3 v) { return v3(v.x * s, v.y * s, v.z * s); }   /* operator*(s, v) */
static double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }  /* ScalarProd :60 */
static V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static double vabs(V3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }   /* abs :71 */

/* ------------------------------------------------------------------ state */
typedef struct {
    double x, y, z, vx, vy, vz, t, w, w0;
    uint32_t cell, pid, draw;
    uint64_t id;
} Part;

typedef struct {
    Part *p;
    uint64_t n, cap;
} Bank;

static int bank_push(Bank *b, const Part *p) {
    if (b->n == b->cap) {
        uint64_t nc = b->cap ? 2 * b->cap : 1024;
        Part *np = (Part *)realloc(b->p, nc * sizeof(Part));
        if (!np) return -1;
        b->p = np;
        b->cap = nc;
    }
    b->p[b->n++] = *p;
    return 0;
}

struct Oracle {
    StormProblemDesc d;
    uint32_t nx, ny, nz;
    uint64_t N;
    double *xe, *ye, *ze, *xc, *yc, *zc;
    double X0, X1, Y0, Y1, Z0, Z1;
    /* cells */
    double *T, *mass, *vol, *eint, *ceint, *sigA, *sigS, *fleck, *rwSigT, *eradAvg, *eradCensus, *emitE;
    double *rhoF;
    uint8_t *rwElig;
    uint64_t *segs, *photons;
    StormBoxFace faces[6];
    /* banks */
    Bank census, bank;
    uint64_t pidLimit;   /* every pid of the current census is below this */
    /* particle shards (orc_set_sharding): S shards, this instance holds [shardLo, shardHi) */
    uint32_t shards, shardLo, shardHi;
    uint64_t *shardCensus;         /* census particles per shard after the last comb (every shard) */
    uint64_t nCenGlobal, nCellEmitGlobal, nFaceEmitGlobal;   /* the current step's global counts */
    double *dep;                   /* this instance's material deposits of the current step */
    StormExchangeFn exchange;
    void *exchangeUser;
    uint32_t step;
    StormStepStats st;
    int32_t derr;
    uint64_t derrCell, derrParticle;
};

static void raise(Oracle *o, int32_t code, uint64_t cell, uint64_t part) {
    if (o->derr == 0) { o->derr = code; o->derrCell = cell; o->derrParticle = part; }
}

static void cell_ijk(const Oracle *o, uint64_t c, uint32_t *i, uint32_t *j, uint32_t *k) {
    *i = (uint32_t)(c % o->nx);
    *j = (uint32_t)((c / o->nx) % o->ny);
    *k = (uint32_t)(c / ((uint64_t)o->nx * o->ny));
}
static V3 center(const Oracle *o, uint64_t c) {
    uint32_t i, j, k;
    cell_ijk(o, c, &i, &j, &k);
    return v3(o->xc[i], o->yc[j], o->zc[k]);
}
static int outside_box(const Oracle *o, V3 p) {   /* Grid::IsPointOutsideBox(point) */
    return p.x < o->X0 || p.x > o->X1 || p.y < o->Y0 || p.y > o->Y1 || p.z < o->Z0 || p.z > o->Z1;
}

/* global face index of side s (0..5, GetCellFaces order) of cell (i,j,k) */
static uint64_t face_index(const Oracle *o, uint32_t i, uint32_t j, uint32_t k, int s) {
    uint64_t nx = o->nx, ny = o->ny, nz = o->nz;
    uint64_t nxf = (nx + 1) * ny * nz, nyf = nx * (ny + 1) * nz;
    switch (s) {
    case 0: return i + (nx + 1) * (j + ny * k);
    case 1: return (i + 1) + (nx + 1) * (j + ny * k);
    case 2: return nxf + i + nx * (j + (ny + 1) * k);
    case 3: return nxf + i + nx * ((j + 1) + (ny + 1) * k);
    case 4: return nxf + nyf + i + nx * (j + ny * k);
    default: return nxf + nyf + i + nx * (j + ny * (k + 1));
    }
}

/* Face data of side s of a cell as updateGridData builds it
 * (physics/MonteCarloPhysics.hpp:60-84): inward unit normal and face centroid. */
static void cell_face(const Oracle *o, uint32_t i, uint32_t j, uint32_t k, int s, V3 *n, V3 *pf) {
    int axis = s / 2, hi = s & 1;
    V3 N = v3(axis == 0 ? 1.0 : 0.0, axis == 1 ? 1.0 : 0.0, axis == 2 ? 1.0 : 0.0);   /* Grid::Normal */
    double fx = axis == 0 ? o->xe[i + hi] : o->xc[i];
    double fy = axis == 1 ? o->ye[j + hi] : o->yc[j];
    double fz = axis == 2 ? o->ze[k + hi] : o->zc[k];
    V3 F = v3(fx, fy, fz);                                                                /* Grid::FaceCM */
    V3 C = v3(o->xc[i], o->yc[j], o->zc[k]);
    if (dot(N, vsub(C, F)) < 0) N = vscale(-1, N);
    double len = vabs(N);
    if (len > 0) N = v3(N.x / len, N.y / len, N.z / len);                                  /* normalize :80-84 */
    *n = N;
    *pf = F;
}

/* neighbour across side s: a cell index, or Ncells + face index for a ghost */
static uint64_t neighbour(const Oracle *o, uint32_t i, uint32_t j, uint32_t k, int s) {
    uint64_t c = i + (uint64_t)o->nx * (j + (uint64_t)o->ny * k);
    switch (s) {
    case 0: if (i > 0) return c - 1; break;
    case 1: if (i + 1 < o->nx) return c + 1; break;
    case 2: if (j > 0) return c - o->nx; break;
    case 3: if (j + 1 < o->ny) return c + o->nx; break;
    case 4: if (k > 0) return c - (uint64_t)o->nx * o->ny; break;
    default: if (k + 1 < o->nz) return c + (uint64_t)o->nx * o->ny; break;
    }
    return o->N + face_index(o, i, j, k, s);
}

/* Particle::distanceToNearestFace (particle/Particle.hpp:188-279) and
 * getIntersectionDetails (physics/MonteCarloPhysics.hpp:86-99).  Returns 0 ok. */
static int intersection(const Oracle *o, const Part *p, double *tFace, uint64_t *next) {
    uint32_t i, j, k;
    cell_ijk(o, p->cell, &i, &j, &k);
    V3 loc = v3(p->x, p->y, p->z), vel = v3(p->vx, p->vy, p->vz);
    double minA = DBL_MAX;
    int minF = -1;
    const double velocityAbs = EPSILON_FACE * vabs(vel);
    for (int s = 0; s < 6; ++s) {
        V3 n, pf;
        cell_face(o, i, j, k, s, &n, &pf);
        double nv = dot(n, vel);
        if (nv >= -velocityAbs) continue;
        double alpha = dot(vsub(pf, loc), n) / nv;
        if (alpha < minA) {
            if (alpha > 0) { minA = alpha; minF = s; }
        }
    }
    if (minA == DBL_MAX) return -1;
    *tFace = minA;
    *next = neighbour(o, i, j, k, minF);
    return 0;
}

/* ------------------------------------------------------------------ Random Walk (radiation/RandomWalk.hpp) */
#define RW_TABLE 1024
#define RW_RADIUS 256
#define RW_XGRID 512
static const double RW_PI = 3.14159265358979323846;
static const double RW_TAU_MIN = 1e-8, RW_TAU_MAX = 64.0, RW_TAU_FREE = 0.01;
static double g_tau[RW_TABLE], g_surv[RW_TABLE];
static double *g_rad = NULL;

static double clampd(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); } /* std::clamp */

static double survival_eigen(double tau) {   /* :178-192 */
    double sum = 0.0;
    for (int n = 1; n <= 500; ++n) {
        double arg = -(double)(n * n) * RW_PI * RW_PI * tau;
        if (arg < -700.0) break;
        double term = exp(arg);
        sum += (n % 2 == 1) ? term : -term;
    }
    return clampd(2.0 * sum, 0.0, 1.0);
}
double orc_rw_survival(double tau) {   /* computeSurvival :139-150 */
    if (tau <= 0.0) return 1.0;
    if (tau < 1e-4) return 1.0;
    return survival_eigen(tau);
}
static double radial_free(double x, double tau) {   /* :194-206 */
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.0;
    double a = x / (2.0 * sqrt(tau));
    return clampd(erf(a) - 2.0 * a * exp(-a * a) / sqrt(RW_PI), 0.0, 1.0);
}
static double radial_eigen(double x, double tau) {   /* :208-237 */
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.0;
    double S = orc_rw_survival(tau);
    if (S < 1e-30) return 1.0;
    double sum = 0.0;
    for (int n = 1; n <= 500; ++n) {
        double arg = -(double)(n * n) * RW_PI * RW_PI * tau;
        if (arg < -700.0) break;
        double npi = (double)n * RW_PI;
        double npx = npi * x;
        double term = exp(arg) * (sin(npx) / npi - x * cos(npx));
        sum += term;
    }
    return clampd(2.0 * sum / S, 0.0, 1.0);
}
double orc_rw_radial_cdf(double x, double tau) {   /* computeRadialCDF :152-167 */
    if (tau <= 0.0) return (x > 0.0) ? 1.0 : 0.0;
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.0;
    return (tau < RW_TAU_FREE) ? radial_free(x, tau) : radial_eigen(x, tau);
}
/* std::lower_bound as libstdc++ implements it (first element for which comp(e, v) is false) */
static size_t lower_bound_asc(const double *a, size_t n, double v) {
    size_t first = 0, count = n;
    while (count > 0) {
        size_t step = count / 2, it = first + step;
        if (a[it] < v) { first = it + 1; count -= step + 1; } else count = step;
    }
    return first;
}
static size_t lower_bound_desc(const double *a, size_t n, double v) {   /* comp(a, b) = a > b */
    size_t first = 0, count = n;
    while (count > 0) {
        size_t step = count / 2, it = first + step;
        if (a[it] > v) { first = it + 1; count -= step + 1; } else count = step;
    }
    return first;
}
static void rw_build(void) {   /* RandomWalk::RandomWalk :23-79 */
    if (g_rad) return;
    g_rad = (double *)malloc(sizeof(double) * RW_TABLE * RW_RADIUS);
    double logMin = log(RW_TAU_MIN), logMax = log(RW_TAU_MAX);
    for (size_t i = 0; i < RW_TABLE; ++i) {
        double frac = (double)i / (double)(RW_TABLE - 1);
        double tau = exp(logMin + frac * (logMax - logMin));
        g_tau[i] = tau;
        g_surv[i] = orc_rw_survival(tau);
    }
    double g[RW_XGRID];
    for (size_t i = 0; i < RW_TABLE; ++i) {
        double tau = g_tau[i];
        for (size_t k = 0; k < RW_XGRID; ++k) g[k] = orc_rw_radial_cdf((double)k / (double)(RW_XGRID - 1), tau);
        for (size_t j = 0; j < RW_RADIUS; ++j) {
            double xi = (double)j / (double)(RW_RADIUS - 1);
            double r;
            if (xi <= g[0]) r = 0.0;
            else if (xi >= g[RW_XGRID - 1]) r = 1.0;
            else {
                size_t idx = lower_bound_asc(g, RW_XGRID, xi);
                if (idx == 0) idx = 1;
                double g0 = g[idx - 1], g1 = g[idx];
                double x0 = (double)(idx - 1) / (double)(RW_XGRID - 1);
                double x1 = (double)idx / (double)(RW_XGRID - 1);
                double f = (g1 > g0) ? (xi - g0) / (g1 - g0) : 0.5;
                r = x0 + f * (x1 - x0);
            }
            g_rad[i * RW_RADIUS + j] = r;
        }
    }
}
void orc_rw_tables(double *tau, double *survival, double *radius) {
    rw_build();
    if (tau) memcpy(tau, g_tau, sizeof(g_tau));
    if (survival) memcpy(survival, g_surv, sizeof(g_surv));
    if (radius) memcpy(radius, g_rad, sizeof(double) * RW_TABLE * RW_RADIUS);
}
double orc_rw_sample_leak(double xi) {   /* sampleLeakTime :81-112 */
    rw_build();
    double target = 1.0 - xi;
    if (target >= g_surv[0]) return g_tau[0];
    if (target <= g_surv[RW_TABLE - 1]) return g_tau[RW_TABLE - 1];
    size_t idx = lower_bound_desc(g_surv, RW_TABLE, target);
    if (idx == 0) return g_tau[0];
    if (idx == RW_TABLE) return g_tau[RW_TABLE - 1];
    double S0 = g_surv[idx - 1], S1 = g_surv[idx];
    double t0 = g_tau[idx - 1], t1 = g_tau[idx];
    double frac = (S0 - target) / (S0 - S1);
    double logT = log(t0) + frac * (log(t1) - log(t0));
    return exp(logT);
}
double orc_rw_sample_radius(double tau, double xi) {   /* sampleRadius :114-137 */
    rw_build();
    double logTau = log(clampd(tau, RW_TAU_MIN, RW_TAU_MAX));
    double logMin = log(RW_TAU_MIN), logMax = log(RW_TAU_MAX);
    double tauPos = (logTau - logMin) / (logMax - logMin) * (double)(RW_TABLE - 1);
    size_t tauIdx = (size_t)tauPos;
    if (tauIdx > RW_TABLE - 2) tauIdx = RW_TABLE - 2;
    double tauFrac = tauPos - (double)tauIdx;
    double xiC = clampd(xi, 0.0, 1.0);
    double xiPos = xiC * (double)(RW_RADIUS - 1);
    size_t xiIdx = (size_t)xiPos;
    if (xiIdx > RW_RADIUS - 2) xiIdx = RW_RADIUS - 2;
    double xiFrac = xiPos - (double)xiIdx;
    double r00 = g_rad[tauIdx * RW_RADIUS + xiIdx];
    double r01 = g_rad[tauIdx * RW_RADIUS + xiIdx + 1];
    double r10 = g_rad[(tauIdx + 1) * RW_RADIUS + xiIdx];
    double r11 = g_rad[(tauIdx + 1) * RW_RADIUS + xiIdx + 1];
    double r0 = r00 + xiFrac * (r01 - r00);
    double r1 = r10 + xiFrac * (r11 - r10);
    return clampd(r0 + tauFrac * (r1 - r0), 0.0, 1.0);
}

/* ------------------------------------------------------------------ samplers */
/* RadiationOpacityModel::isotropicVelocity (radiation/RadiationOpacityModel.hpp:139-150) */
static V3 isotropic(Rng *r, double clight) {
    const double twoPi = 6.283185307179586476925286766559;
    double theta = twoPi * rng_raw(r);
    double cosTheta = 2.0 * rng_raw(r) - 1.0;
    double s2 = 1.0 - cosTheta * cosTheta;
    if (s2 < 0.0) s2 = 0.0;
    double sinTheta = sqrt(s2);
    return v3(sinTheta * cos(theta) * clight, sinTheta * sin(theta) * clight, cosTheta * clight);
}
void orc_isotropic(const double *tape2, double clight, double *out3) {
    Rng r;
    memset(&r, 0, sizeof(r));
    r.tape_mode = 1; r.tape = tape2; r.len = 2;
    V3 v = isotropic(&r, clight);
    out3[0] = v.x; out3[1] = v.y; out3[2] = v.z;
}

/* Vertex coordinates of side s of cell (i,j,k) in GetPointsInFace order. */
static void face_vertices(const Oracle *o, uint32_t i, uint32_t j, uint32_t k, int s, V3 q[4]) {
    int axis = s / 2, hi = s & 1;
    if (axis == 0) {
        double X = o->xe[i + hi];
        q[0] = v3(X, o->ye[j], o->ze[k]); q[1] = v3(X, o->ye[j + 1], o->ze[k]);
        q[2] = v3(X, o->ye[j + 1], o->ze[k + 1]); q[3] = v3(X, o->ye[j], o->ze[k + 1]);
    } else if (axis == 1) {
        double Y = o->ye[j + hi];
        q[0] = v3(o->xe[i], Y, o->ze[k]); q[1] = v3(o->xe[i], Y, o->ze[k + 1]);
        q[2] = v3(o->xe[i + 1], Y, o->ze[k + 1]); q[3] = v3(o->xe[i + 1], Y, o->ze[k]);
    } else {
        double Z = o->ze[k + hi];
        q[0] = v3(o->xe[i], o->ye[j], Z); q[1] = v3(o->xe[i + 1], o->ye[j], Z);
        q[2] = v3(o->xe[i + 1], o->ye[j + 1], Z); q[3] = v3(o->xe[i], o->ye[j + 1], Z);
    }
}

/* RandomInCellPositionSampler::operator() (utils/RandomInCell.hpp:11-67) */
static V3 sample_in_cell(const Oracle *o, uint64_t cell, Rng *r) {
    uint32_t i, j, k;
    cell_ijk(o, cell, &i, &j, &k);
    V3 c = center(o, cell);
    double cum[12];
    V3 tri[12][3];
    double total = 0;
    int nt = 0;
    for (int s = 0; s < 6; ++s) {
        V3 q[4];
        face_vertices(o, i, j, k, s, q);
        for (int t = 1; t + 1 < 4; ++t) {
            V3 a = vsub(q[0], c), b = vsub(q[t], c), cc = vsub(q[t + 1], c);
            double vol = fabs(dot(a, cross(b, cc)));
            total += vol;
            cum[nt] = total;
            tri[nt][0] = q[0]; tri[nt][1] = q[t]; tri[nt][2] = q[t + 1];
            ++nt;
        }
    }
    double rr = rng_raw(r) * total;
    size_t idx = lower_bound_asc(cum, (size_t)nt, rr);
    if (idx >= (size_t)nt) idx = (size_t)nt - 1;
    double s = rng_raw(r), t = rng_raw(r), u = rng_raw(r), tmp;
    if (s > t) { tmp = s; s = t; t = tmp; }
    if (t > u) { tmp = t; t = u; u = tmp; }
    if (s > t) { tmp = s; s = t; t = tmp; }
    V3 *tv = tri[idx];
    return vadd(vadd(vadd(vscale(s, tv[0]), vscale(t - s, tv[1])), vscale(u - t, tv[2])), vscale(1 - u, c));
}
int orc_sample_in_cell(Oracle *o, uint32_t cell, const double *tape4, double *out3) {
    Rng r;
    memset(&r, 0, sizeof(r));
    r.tape_mode = 1; r.tape = tape4; r.len = 4;
    V3 p = sample_in_cell(o, cell, &r);
    out3[0] = p.x; out3[1] = p.y; out3[2] = p.z;
    return 0;
}

/* RandomPointOnFace (utils/RandomOnFace.hpp:15-66) for the face given by
 * its vertices (4, in GetPointsInFace order). */
static V3 point_on_face(const V3 q[4], Rng *r) {
    double cum[2];
    double total = 0;
    for (int t = 1; t + 1 < 4; ++t) {
        double area = vabs(cross(vsub(q[t], q[0]), vsub(q[t + 1], q[0])));
        total += area;
        cum[t - 1] = total;
    }
    double rr = rng_raw(r) * total;
    size_t idx = lower_bound_asc(cum, 2, rr);
    if (idx >= 2) idx = 1;
    double r1 = rng_raw(r), r2 = rng_raw(r);
    if (r1 + r2 > 1) { r1 = 1 - r1; r2 = 1 - r2; }
    V3 a = q[0], b = q[idx + 1], c = q[idx + 2];
    return vadd(vadd(vscale(1 - r1 - r2, a), vscale(r1, b)), vscale(r2, c));
}
/* face -> (cell, side): the grid's global face numbering */
static int face_to_cell_side(const Oracle *o, uint64_t f, uint32_t *i, uint32_t *j, uint32_t *k, int *s) {
    uint64_t nx = o->nx, ny = o->ny, nz = o->nz;
    uint64_t nxf = (nx + 1) * ny * nz, nyf = nx * (ny + 1) * nz;
    if (f < nxf) {
        uint64_t ii = f % (nx + 1), jj = (f / (nx + 1)) % ny, kk = f / ((nx + 1) * ny);
        if (ii < nx) { *i = (uint32_t)ii; *s = 0; } else { *i = (uint32_t)(ii - 1); *s = 1; }
        *j = (uint32_t)jj; *k = (uint32_t)kk;
        return 0;
    }
    f -= nxf;
    if (f < nyf) {
        uint64_t ii = f % nx, jj = (f / nx) % (ny + 1), kk = f / (nx * (ny + 1));
        if (jj < ny) { *j = (uint32_t)jj; *s = 2; } else { *j = (uint32_t)(jj - 1); *s = 3; }
        *i = (uint32_t)ii; *k = (uint32_t)kk;
        return 0;
    }
    f -= nyf;
    uint64_t ii = f % nx, jj = (f / nx) % ny, kk = f / (nx * ny);
    if (kk < nz) { *k = (uint32_t)kk; *s = 4; } else { *k = (uint32_t)(kk - 1); *s = 5; }
    *i = (uint32_t)ii; *j = (uint32_t)jj;
    return 0;
}
int orc_point_on_face(Oracle *o, uint64_t face, const double *tape3, double *out3) {
    uint32_t i, j, k;
    int s;
    face_to_cell_side(o, face, &i, &j, &k, &s);
    V3 q[4];
    face_vertices(o, i, j, k, s, q);
    Rng r;
    memset(&r, 0, sizeof(r));
    r.tape_mode = 1; r.tape = tape3; r.len = 3;
    V3 p = point_on_face(q, &r);
    out3[0] = p.x; out3[1] = p.y; out3[2] = p.z;
    return 0;
}

/* ------------------------------------------------------------------ boundary (boundary/BoundaryCondition.hpp:61-108) */
static void box_face_vertices(const Oracle *o, int f, V3 q[4]) {
    double X0 = o->X0, X1 = o->X1, Y0 = o->Y0, Y1 = o->Y1, Z0 = o->Z0, Z1 = o->Z1;
    switch (f) {
    case 0: q[0] = v3(X0, Y0, Z0); q[1] = v3(X0, Y1, Z0); q[2] = v3(X0, Y1, Z1); q[3] = v3(X0, Y0, Z1); break;
    case 1: q[0] = v3(X1, Y0, Z0); q[1] = v3(X1, Y1, Z0); q[2] = v3(X1, Y1, Z1); q[3] = v3(X1, Y0, Z1); break;
    case 2: q[0] = v3(X0, Y0, Z0); q[1] = v3(X0, Y0, Z1); q[2] = v3(X1, Y0, Z1); q[3] = v3(X1, Y0, Z0); break;
    case 3: q[0] = v3(X0, Y1, Z0); q[1] = v3(X0, Y1, Z1); q[2] = v3(X1, Y1, Z1); q[3] = v3(X1, Y1, Z0); break;
    case 4: q[0] = v3(X0, Y0, Z0); q[1] = v3(X1, Y0, Z0); q[2] = v3(X1, Y1, Z0); q[3] = v3(X0, Y1, Z0); break;
    default: q[0] = v3(X0, Y0, Z1); q[1] = v3(X1, Y0, Z1); q[2] = v3(X1, Y1, Z1); q[3] = v3(X0, Y1, Z1); break;
    }
}
/* getInwardBoxFaceNormalIfClose :61-85 */
static int box_face_close(const Oracle *o, int f, V3 loc, V3 *normal, double *faceScale) {
    V3 q[4];
    box_face_vertices(o, f, q);
    V3 onFace = q[0];
    V3 u = vsub(q[1], q[0]), v = vsub(q[2], q[0]);
    V3 n = cross(u, v);
    double au = vabs(u), av = vabs(v);
    double fs = (av < au) ? av : au;   /* std::min */
    double nn = vabs(n);
    if (!(nn > 0.0) || !isfinite(nn) || !(fs > 0.0) || !isfinite(fs)) return 0;
    double pd = dot(n, vsub(loc, onFace));
    if (fabs(pd) >= EPSILON_FACE * fs * fs * fs) return 0;
    n = vscale(1.0 / nn, n);
    V3 boxCenter = vscale(0.5, vadd(v3(o->X0, o->Y0, o->Z0), v3(o->X1, o->Y1, o->Z1)));
    if (dot(n, vsub(boxCenter, onFace)) < 0.0) n = vscale(-1.0, n);
    *normal = n;
    *faceScale = fs;
    return 1;
}
/* reflectParticleOnBoxFace :87-108 */
static int reflect_box_face(const Oracle *o, int f, Part *p) {
    V3 n;
    double fs;
    V3 loc = v3(p->x, p->y, p->z);
    if (!box_face_close(o, f, loc, &n, &fs)) return 0;
    V3 q[4];
    box_face_vertices(o, f, q);
    double sd = dot(vsub(loc, q[0]), n);
    V3 d = vscale(sd, n);
    loc = vsub(loc, d);
    double sc = REFLECT_NUDGE * fs;
    loc = vadd(loc, vscale(sc, n));
    p->x = loc.x; p->y = loc.y; p->z = loc.z;
    V3 vel = v3(p->vx, p->vy, p->vz);
    double vn = dot(vel, n);
    if (vn < 0.0) {
        double s2 = 2.0 * vn;
        vel = vsub(vel, vscale(s2, n));
        p->vx = vel.x; p->vy = vel.y; p->vz = vel.z;
    }
    return 1;
}
/* BoundaryCondition::apply for the per-face descriptor (VacuumBoundary :18-22,
 * RigidBoundary :43-58, SideTemperature :84-112, TwoSidesTemperature :97-123). */
static int boundary_apply(Oracle *o, Part *p) {
    if (o->d.escape_without_check) return REMOVE;
    int status = DONE;
    for (int f = 0; f < 6; ++f) {
        V3 n;
        double fs;
        if (box_face_close(o, f, v3(p->x, p->y, p->z), &n, &fs)) {
            if (o->faces[f].action == STORM_FACE_ESCAPE) return REMOVE;
            if (reflect_box_face(o, f, p)) status = REFLECT;
        }
    }
    return status;
}

/* ------------------------------------------------------------------ physics step */
typedef struct {
    int status;       /* ParticleStatus */
    uint64_t next;
    double dmat, derad;
    int usedRW;
    int error;
} StepOut;

static int try_random_walk(Oracle *o, Part *p, Rng *r, StepOut *so) {   /* RadiationIMC.hpp:1065-1276 (gray) */
    uint32_t i, j, k;
    const uint64_t cell = p->cell;
    cell_ijk(o, cell, &i, &j, &k);
    V3 loc = v3(p->x, p->y, p->z);
    double Ro = DBL_MAX;   /* computeMinDistanceToFaces :956-969 */
    for (int s = 0; s < 6; ++s) {
        V3 n, pf;
        cell_face(o, i, j, k, s, &n, &pf);
        double d = dot(vsub(loc, pf), n);
        Ro = (d < Ro) ? d : Ro;
    }
    Ro = (Ro > 0.0) ? Ro : 0.0;
    const double c = o->d.clight;
    double sigmaT = o->rwSigT[cell];
    double sigma_a_eff = o->sigA[cell];
    double D_phys = (sigmaT > 0.0) ? c / (3.0 * sigmaT) : 0.0;
    int doRW = (Ro > 0.0 && sigmaT > 0.0 && D_phys > 0.0 && Ro * sigmaT >= o->d.rw_min_particle_optical_depth);
    if (!doRW) return 0;
    double f = o->fleck[cell];
    double tauLeak = orc_rw_sample_leak(rng_open(r));
    double tLeak = tauLeak * Ro * Ro / D_phys;
    double tCensus = p->t;
    double tUp = DBL_MAX;
    int ev;   /* 0 leak, 1 census, 2 upscatter */
    double dt;
    if (tLeak <= tCensus && tLeak <= tUp) { ev = 0; dt = tLeak; }
    else if (tCensus <= tUp) { ev = 1; dt = tCensus; }
    else { ev = 2; dt = tUp; }
    double rwAbsRate = sigma_a_eff * f * c;
    double rwExp = expm1(-dt * rwAbsRate);
    if (!o->d.no_hydro_feedback) so->dmat += -rwExp * p->w;
    if (rwAbsRate > 0.0) so->derad += p->w * rwExp * (-1.0 / rwAbsRate);
    p->w *= 1.0 + rwExp;
    p->t -= dt;
    so->usedRW = 1;
    if (fabs(p->w) < p->w0 * 1e-4) {
        so->status = REMOVE;
        if (!o->d.no_hydro_feedback) so->dmat += p->w;
        return 1;
    }
    double cosTheta = 2.0 * rng_open(r) - 1.0;
    double s2 = 1.0 - cosTheta * cosTheta;
    double sinTheta = sqrt(s2 > 0.0 ? s2 : 0.0);
    double phi = 2.0 * RW_PI * rng_open(r);
    V3 posDir = v3(sinTheta * cos(phi), sinTheta * sin(phi), cosTheta);
    double disp;
    if (ev == 0) disp = Ro;
    else {
        double tauPos = D_phys * dt / (Ro * Ro);
        disp = Ro * orc_rw_sample_radius(tauPos, rng_open(r));
    }
    if (disp > Ro * (1.0 + 1e-12)) disp = Ro;
    V3 rwCenter = loc;
    loc = vadd(rwCenter, vscale(disp, posDir));
    V3 mc = center(o, cell);
    loc = vadd(vscale(1.0 - RW_NUDGE, loc), vscale(RW_NUDGE, mc));
    int guard = 0;
    for (int s = 0; s < 6; ++s) {
        V3 n, pf;
        cell_face(o, i, j, k, s, &n, &pf);
        double d = dot(vsub(loc, pf), n);
        if (d < 0.0) {
            disp *= 0.99;
            loc = vadd(rwCenter, vscale(disp, posDir));
            s = -1;
            if (++guard > 100000) { so->error = STORM_DERR_RW_SHRINK; return 1; }
        }
    }
    p->x = loc.x; p->y = loc.y; p->z = loc.z;
    V3 vel = isotropic(r, c);
    p->vx = vel.x; p->vy = vel.y; p->vz = vel.z;
    so->status = (ev == 1) ? DONE : NO_CELL_MOVE;
    return 1;
}

/* RadiationIMC::step (radiation/RadiationIMC.hpp:1700-1881), gray, no hydro. */
static void physics_step(Oracle *o, Part *p, Rng *r, StepOut *so) {
    memset(so, 0, sizeof(*so));
    so->next = UINT64_MAX;
    so->status = NO_CELL_MOVE;
    const uint64_t cell = p->cell;
    double tFace;
    uint64_t next;
    if (intersection(o, p, &tFace, &next) != 0) { so->error = STORM_DERR_NO_FACE; return; }
    if (o->d.with_random_walk && o->rwElig[cell]) {
        if (try_random_walk(o, p, r, so)) return;
    }
    const double c = o->d.clight;
    double absorptionOpacity = o->sigA[cell];
    double elasticScatteringOpacity = o->sigS[cell];
    double effectiveAbsorptionOpacity = (1.0 - o->fleck[cell]) * absorptionOpacity;
    double eventOpacity = elasticScatteringOpacity + effectiveAbsorptionOpacity;
    double scatteringLength = (eventOpacity > 0.0) ? 1.0 / eventOpacity : INFINITY;
    double lp = -log1p(rng_open(r) - 1.0);
    double scatteringDistance = scatteringLength * lp / 1.0;
    double speed = vabs(v3(p->vx, p->vy, p->vz));
    double timeScattering = isfinite(scatteringDistance) ? scatteringDistance / speed : INFINITY;
    double times[3] = {tFace, timeScattering, p->t};
    int best = 0;   /* std::min_element: first smallest */
    for (int q = 1; q < 3; ++q) if (times[q] < times[best]) best = q;
    double dt = times[best];
    p->t -= dt;
    double weightEvolutionOpacity = absorptionOpacity * o->fleck[cell];
    double tmp2 = weightEvolutionOpacity * c;
    double tmp = -dt * tmp2;
    double expFactor1 = expm1(tmp * 1.0);
    double expFactor2 = expm1(tmp);
    double integratedForTally = p->w * dt;
    if (fabs(tmp2 * dt) >= 1e-12) integratedForTally = p->w * expFactor2 * (-1.0 / tmp2);
    p->x += p->vx * dt;
    p->y += p->vy * dt;
    p->z += p->vz * dt;
    if (!o->d.no_hydro_feedback) so->dmat += -expFactor2 * p->w;
    so->derad += integratedForTally;
    p->w *= 1.0 + expFactor1;
    if (fabs(p->w) < p->w0 * 1e-3) {
        so->status = REMOVE;
        if (!o->d.no_hydro_feedback) so->dmat += p->w;
        return;
    }
    if (best == 0) {
        so->status = CELL_MOVE;
        so->next = next;
    } else if (best == 1) {
        (void)(rng_open(r) * eventOpacity);   /* event-type draw; both branches re-scatter isotropically */
        V3 vel = isotropic(r, c);
        p->vx = vel.x; p->vy = vel.y; p->vz = vel.z;
        so->status = NO_CELL_MOVE;
    } else {
        so->status = DONE;
    }
}

/* manager face / boundary handling (manager/MonteCarloManagerSerial.hpp:318-369).
 * Returns 0 continue, 1 census, 2 removed (cutoff), 3 escaped, -1 error. */
static int manager_handle(Oracle *o, Part *p, const StepOut *so) {
    if (so->status == CELL_MOVE) {
        if (so->next < o->N) {
            V3 c = center(o, so->next);
            V3 l = vadd(vscale(1 - MONTECARLO_EPS, v3(p->x, p->y, p->z)), vscale(MONTECARLO_EPS, c));
            p->x = l.x; p->y = l.y; p->z = l.z;
            p->cell = (uint32_t)so->next;
            return 0;
        }
        int st = boundary_apply(o, p);
        if (st == REFLECT) {
            V3 c = center(o, p->cell);
            V3 l = vadd(vscale(1 - MONTECARLO_EPS, v3(p->x, p->y, p->z)), vscale(MONTECARLO_EPS, c));
            p->x = l.x; p->y = l.y; p->z = l.z;
            return 0;
        }
        if (st == REMOVE) return 3;
        return -1;
    }
    if (so->status == REMOVE) return 2;
    if (so->status == DONE) return 1;
    return 0;
}

/* ------------------------------------------------------------------ lifecycle */
static double *dup(const double *src, uint64_t n, double fill) {
    double *p = (double *)malloc(sizeof(double) * (n ? n : 1));
    for (uint64_t i = 0; i < n; ++i) p[i] = src ? src[i] : fill;
    return p;
}

Oracle *orc_create(const StormProblemDesc *d) {
    Oracle *o = (Oracle *)calloc(1, sizeof(Oracle));
    o->d = *d;
    o->nx = d->nx; o->ny = d->ny; o->nz = d->nz;
    o->N = (uint64_t)d->nx * d->ny * d->nz;
    uint64_t N = o->N;
    o->xe = dup(d->x_edges, d->nx + 1, 0); o->ye = dup(d->y_edges, d->ny + 1, 0); o->ze = dup(d->z_edges, d->nz + 1, 0);
    o->xc = dup(NULL, d->nx, 0); o->yc = dup(NULL, d->ny, 0); o->zc = dup(NULL, d->nz, 0);
    for (uint32_t i = 0; i < d->nx; ++i) o->xc[i] = 0.5 * (o->xe[i] + o->xe[i + 1]);
    for (uint32_t j = 0; j < d->ny; ++j) o->yc[j] = 0.5 * (o->ye[j] + o->ye[j + 1]);
    for (uint32_t k = 0; k < d->nz; ++k) o->zc[k] = 0.5 * (o->ze[k] + o->ze[k + 1]);
    o->X0 = o->xe[0]; o->X1 = o->xe[d->nx]; o->Y0 = o->ye[0]; o->Y1 = o->ye[d->ny]; o->Z0 = o->ze[0]; o->Z1 = o->ze[d->nz];
    o->T = dup(d->temperature, N, 0);
    o->mass = dup(d->mass, N, 0);
    o->eint = dup(d->internal_energy, N, 0);
    o->ceint = dup(d->cell_internal_energy ? d->cell_internal_energy : d->internal_energy, N, 0);
    o->vol = dup(NULL, N, 0);
    for (uint64_t c = 0; c < N; ++c) {
        uint32_t i, j, k;
        cell_ijk(o, c, &i, &j, &k);
        o->vol[c] = (o->xe[i + 1] - o->xe[i]) * (o->ye[j + 1] - o->ye[j]) * (o->ze[k + 1] - o->ze[k]);
    }
    o->sigA = dup(d->opacity_kind == STORM_OPACITY_CELL_TABLE ? d->sigma_a : NULL, N, 0);
    o->sigS = dup(d->opacity_kind == STORM_OPACITY_CELL_TABLE ? d->sigma_s : NULL, N, 0);
    o->rhoF = dup(d->density_factor, N, 1.0);
    o->fleck = dup(NULL, N, 1.0);
    o->rwSigT = dup(NULL, N, 0);
    o->eradAvg = dup(NULL, N, 0);
    o->eradCensus = dup(NULL, N, 0);
    o->emitE = dup(NULL, N, 0);
    o->rwElig = (uint8_t *)calloc(N ? N : 1, 1);
    o->segs = (uint64_t *)calloc(N ? N : 1, sizeof(uint64_t));
    o->photons = (uint64_t *)calloc(N ? N : 1, sizeof(uint64_t));
    memcpy(o->faces, d->faces, sizeof(o->faces));
    o->d.x_edges = o->d.y_edges = o->d.z_edges = NULL;
    o->d.temperature = o->d.mass = o->d.internal_energy = o->d.cell_internal_energy = NULL;
    o->d.sigma_a = o->d.sigma_s = o->d.density_factor = NULL;
    if (d->with_random_walk) rw_build();
    o->shards = 1; o->shardLo = 0; o->shardHi = 1;
    return o;
}

int orc_set_sharding(Oracle *o, uint32_t shards, uint32_t lo, uint32_t hi, StormExchangeFn exchange, void *user) {
    if (!o || shards == 0 || lo >= hi || hi > shards || o->census.n || !o->d.comb_enabled ||
        o->d.comb_kind != STORM_COMB_PLAIN)
        return -1;
    o->shards = shards; o->shardLo = lo; o->shardHi = hi;
    free(o->shardCensus);
    o->shardCensus = (uint64_t *)calloc(shards, sizeof(uint64_t));
    free(o->dep);
    o->dep = dup(NULL, o->N, 0);
    o->exchange = exchange;
    o->exchangeUser = user;
    return 0;
}

/* the exchange: an in-place sum over every rank (identity without a callback) */
static int exchange_sum(Oracle *o, double *v, uint64_t n) {
    if (!o->exchange) return 0;
    return o->exchange(o->exchangeUser, v, n, NULL) ? -1 : 0;
}

/* first index of shard s when `n` items are cut into S contiguous shards */
static uint64_t shard_begin(uint64_t n, uint32_t s, uint32_t S) {
    return (uint64_t)(((unsigned __int128)n * s) / S);
}

/* census particles of the shards below s (their pids start at this offset) */
static uint64_t census_offset(const Oracle *o, uint32_t s) {
    uint64_t off = 0;
    for (uint32_t q = 0; q < s; ++q) off += o->shardCensus[q];
    return off;
}

/* The shard a pid belongs to: census pids [0, nCen) by the shards' census
 * counts, then cell packets and face packets each cut into S equal ranges. */
static uint32_t shard_of_pid(const Oracle *o, uint64_t pid) {
    const uint32_t S = o->shards;
    if (pid < o->nCenGlobal) {
        uint64_t off = 0;
        for (uint32_t s = 0; s < S; ++s) {
            off += o->shardCensus[s];
            if (pid < off) return s;
        }
        return S - 1;
    }
    uint64_t e = pid - o->nCenGlobal, n = o->nCellEmitGlobal;
    if (e >= n) { e -= n; n = o->nFaceEmitGlobal; }
    uint32_t s = 0;
    while (s + 1 < S && shard_begin(n, s + 1, S) <= e) ++s;
    return s;
}

void orc_destroy(Oracle *o) {
    if (!o) return;
    double *arrs[] = {o->xe, o->ye, o->ze, o->xc, o->yc, o->zc, o->T, o->mass, o->eint, o->ceint, o->vol, o->sigA,
                      o->sigS, o->rhoF, o->fleck, o->rwSigT, o->eradAvg, o->eradCensus, o->emitE};
    for (size_t q = 0; q < sizeof(arrs) / sizeof(arrs[0]); ++q) free(arrs[q]);
    free(o->rwElig); free(o->segs); free(o->photons);
    free(o->census.p); free(o->bank.p);
    free(o->shardCensus); free(o->dep);
    free(o);
}

/* ------------------------------------------------------------------ phases */
/* manager step() start (manager/MonteCarloManagerSerial.hpp:391-405): census
 * particles get timeLeft = dt, initialWeight = |w|, steps = 0, and become the
 * head of the transport bank (pid = position). */
int orc_phase_begin(Oracle *o, double dt) {
    memset(&o->st, 0, sizeof(o->st));
    o->derr = 0;
    o->bank.n = 0;
    /* sharded: this instance's census holds the global pids from the offset of its first shard */
    const uint64_t pid0 = o->shards > 1 ? census_offset(o, o->shardLo) : 0;
    o->nCenGlobal = o->shards > 1 ? census_offset(o, o->shards) : o->census.n;
    for (uint64_t q = 0; q < o->census.n; ++q) {
        Part p = o->census.p[q];
        p.t = dt;
        p.w0 = fabs(p.w);
        p.pid = (uint32_t)(pid0 + q);
        p.draw = 0;
        o->st.energy_census_in += p.w;
        bank_push(&o->bank, &p);
    }
    o->st.census_in = o->census.n;
    o->census.n = 0;
    return 0;
}

/* Opacity plug-in evaluated per cell (CalcPlanckOpacity / CalcScatteringOpacity). */
static void opacity_eval(Oracle *o, uint64_t c, double *sa, double *ss) {
    if (o->d.opacity_kind == STORM_OPACITY_CELL_TABLE) { *sa = o->sigA[c]; *ss = o->sigS[c]; return; }
    double tmax = o->T[c] > o->d.t_floor ? o->T[c] : o->d.t_floor;
    double tf = pow(o->d.kev_kelvin / tmax, o->d.alpha);
    double k = o->d.kP0 * tf * o->rhoF[c];
    *sa = (o->d.cap > 0.0) ? (k < o->d.cap ? k : o->d.cap) : k;
    if (!(o->d.kR0 > 0.0)) { *ss = 0.0; return; }
    double kR = o->d.kR0 * tf * o->rhoF[c];
    double kP = o->d.kP0 * tf * o->rhoF[c];
    double sd = kR - kP;
    *ss = sd > 0.0 ? sd : 0.0;
}
/* EOS::dT2cv */
static double eos_cv(const Oracle *o, uint64_t c) {
    if (o->d.eos_kind == STORM_EOS_LINEAR) return o->d.cv_per_mass;
    double rho = o->mass[c] / o->vol[c];
    double Tm = o->T[c] > 1.0 ? o->T[c] : 1.0;
    double cvVol = o->d.eos_f * o->d.eos_beta * pow(Tm, o->d.eos_beta - 1.0) * pow(rho, 1.0 - o->d.eos_mu);
    return cvVol / rho;
}
/* EOS::de2T */
static double eos_T(const Oracle *o, double rho, double spec) {
    if (o->d.eos_kind == STORM_EOS_LINEAR) return (o->d.cv_per_mass > 0.0) ? spec / o->d.cv_per_mass : 0.0;
    double ev = spec * rho;
    double rf = pow(rho, 1.0 - o->d.eos_mu);
    double ratio = (ev > 0.0 ? ev : 0.0) / (o->d.eos_f * rf);
    return pow(ratio > 0.0 ? ratio : 0.0, 1.0 / o->d.eos_beta);
}

/* RadiationIMC::preStep minus emission (radiation/RadiationIMC.hpp:1618-1672)
 * and precomputeRandomWalkData (:982-1063, gray branch). */
int orc_phase_prestep(Oracle *o, double dt) {
    const double c = o->d.clight, a = o->d.arad;
    for (uint64_t i = 0; i < o->N; ++i) {
        double sa, ss;
        opacity_eval(o, i, &sa, &ss);
        o->sigA[i] = sa;
        o->sigS[i] = ss;
        o->eradAvg[i] = 0.0;
        double cv = eos_cv(o, i);
        double T = o->T[i];
        double T3 = (T * T) * T;   /* boost::math::pow<3> */
        o->fleck[i] = 1.0 / (1.0 + (4.0 * a * T3 * sa * c * dt * 1.0) / cv);
        if (o->fleck[i] < 0.0 || o->fleck[i] > 1.0) raise(o, STORM_DERR_FLECK, i, 0);
        if (o->d.with_random_walk) {
            double sigmaT = sa + ss;
            o->rwSigT[i] = sigmaT;
            uint32_t ii, jj, kk;
            cell_ijk(o, i, &ii, &jj, &kk);
            /* computeCellSurfaceArea: the six face areas in GetCellFaces order */
            double dx = o->xe[ii + 1] - o->xe[ii], dy = o->ye[jj + 1] - o->ye[jj], dz = o->ze[kk + 1] - o->ze[kk];
            double ax = dy * dz, ay = dz * dx, az = dx * dy;
            double S = 0.0;
            S += ax; S += ax; S += ay; S += ay; S += az; S += az;
            double chord = (S > 0.0) ? 4.0 * o->vol[i] / S : 0.0;
            o->rwElig[i] = (sigmaT * chord >= o->d.rw_min_cell_optical_depth);
        }
    }
    return o->derr ? -1 : 0;
}

static void repair_outside(Oracle *o, Part *p, V3 meshPoint, double t0) {
    V3 loc = v3(p->x, p->y, p->z);
    if (!outside_box(o, loc)) return;
    V3 original = loc, direction = vsub(meshPoint, original);
    double t = t0;
    while (outside_box(o, loc) && t < 1.0) {
        loc = vadd(original, vscale(t, direction));
        t *= 2;
    }
    loc = vadd(loc, vscale(1e-8, vsub(meshPoint, loc)));
    p->x = loc.x; p->y = loc.y; p->z = loc.z;
}

/* generateParticles (radiation/RadiationIMC.hpp:2035-2510, gray path) and the
 * per-face boundary source (boundary/SideTemperature.hpp:114-163). */
int orc_phase_emit(Oracle *o, double dt) {
    const double c = o->d.clight, a = o->d.arad;
    const uint64_t N = o->N;
    const uint64_t n = o->d.new_photons_per_cell;
    double total = 0.0;
    for (uint64_t i = 0; i < N; ++i) {
        double T = o->T[i];
        double T4 = (T * T) * (T * T);   /* boost::math::pow<4> */
        o->emitE[i] = o->fleck[i] * o->vol[i] * a * T4 * o->sigA[i] * dt * c;
        total += o->emitE[i];
    }
    uint64_t totalParticles = N * n * 10;
    for (uint64_t i = 0; i < N; ++i) {
        uint64_t share = (total > 0) ? (uint64_t)(o->emitE[i] / total * (double)totalParticles) : n;
        uint64_t cap = n * 20;
        uint64_t m = share < cap ? share : cap;
        o->photons[i] = o->emitE[i] > 0.0 ? (m > n ? m : n) : 0;
    }
    /* packets are numbered globally: cell packet e has pid nCen + e and face
     * packet f has pid nCen + nE + f; a sharded instance keeps the packets of
     * its shards' ranges of each numbering */
    uint64_t nE = 0, nF = 0;
    for (uint64_t i = 0; i < N; ++i) nE += o->photons[i];
    for (uint64_t i = 0; i < N; ++i) {
        uint32_t ii, jj, kk;
        cell_ijk(o, i, &ii, &jj, &kk);
        for (int s = 0; s < 6; ++s)
            if (neighbour(o, ii, jj, kk, s) >= N && o->faces[s].source_temperature > 0.0)
                nF += o->faces[s].packets_per_face;
    }
    o->nCellEmitGlobal = nE;
    o->nFaceEmitGlobal = nF;
    const uint64_t eLo = shard_begin(nE, o->shardLo, o->shards), eHi = shard_begin(nE, o->shardHi, o->shards);
    const uint64_t fLo = shard_begin(nF, o->shardLo, o->shards), fHi = shard_begin(nF, o->shardHi, o->shards);
    const uint64_t pidBase = o->nCenGlobal;
    uint64_t e = 0;
    for (uint64_t i = 0; i < N; ++i) {
        uint64_t np = o->photons[i];
        if (np == 0) continue;
        double E = o->emitE[i];
        if (!o->d.no_hydro_feedback) o->eint[i] -= E;
        o->st.energy_emission_debit += E;
        double energyPerPhoton = E * 1.0 / (double)np;
        V3 mc = center(o, i);
        for (uint64_t q = 0; q < np; ++q, ++e) {
            if (e < eLo || e >= eHi) continue;
            Rng r;
            memset(&r, 0, sizeof(r));
            r.seed = o->d.seed; r.tag = TAG_CELL_EMIT; r.step = o->step; r.pid = (uint32_t)e;
            Part p;
            memset(&p, 0, sizeof(p));
            p.cell = (uint32_t)i;
            V3 loc = sample_in_cell(o, i, &r);
            p.x = loc.x; p.y = loc.y; p.z = loc.z;
            repair_outside(o, &p, mc, 1e-8);
            V3 v = isotropic(&r, c);
            p.vx = v.x; p.vy = v.y; p.vz = v.z;
            p.t = dt * rng_open(&r);
            p.w = energyPerPhoton;
            p.w0 = fabs(p.w);
            p.pid = (uint32_t)(pidBase + e);
            p.draw = 0;
            o->st.energy_emitted += p.w;
            bank_push(&o->bank, &p);
        }
    }
    o->st.emitted_cells = eHi - eLo;
    /* face sources: cells in index order, sides in GetCellFaces order */
    uint64_t fpk = 0;
    for (uint64_t i = 0; i < N; ++i) {
        uint32_t ii, jj, kk;
        cell_ijk(o, i, &ii, &jj, &kk);
        for (int s = 0; s < 6; ++s) {
            uint64_t nb = neighbour(o, ii, jj, kk, s);
            if (nb < N) continue;
            const StormBoxFace *bf = &o->faces[s];
            if (!(bf->source_temperature > 0.0) || bf->packets_per_face == 0) continue;
            int axis = s / 2;
            double sgn = (s & 1) ? -1.0 : 1.0;
            uint64_t Np = bf->packets_per_face;
            double Tf = bf->source_temperature;
            double T4 = (Tf * Tf) * (Tf * Tf);
            uint32_t a1 = ii, a2 = jj, a3 = kk;
            (void)a1; (void)a2; (void)a3;
            double dx = o->xe[ii + 1] - o->xe[ii], dy = o->ye[jj + 1] - o->ye[jj], dz = o->ze[kk + 1] - o->ze[kk];
            double area = axis == 0 ? dy * dz : (axis == 1 ? dz * dx : dx * dy);   /* Grid::GetArea */
            double energyToProduce = o->d.sigma_sb * T4 * area * dt / (double)Np;
            V3 q4[4];
            face_vertices(o, ii, jj, kk, s, q4);
            V3 mc = center(o, i);
            for (uint64_t q = 0; q < Np; ++q, ++fpk) {
                if (fpk < fLo || fpk >= fHi) continue;
                Rng r;
                memset(&r, 0, sizeof(r));
                r.seed = o->d.seed; r.tag = TAG_FACE_EMIT; r.step = o->step; r.pid = (uint32_t)fpk;
                Part p;
                memset(&p, 0, sizeof(p));
                V3 loc = point_on_face(q4, &r);
                double mu = sqrt(rng_raw(&r));
                double vv[3];
                vv[axis] = sgn * mu;
                double _1mmu = sqrt(1 - mu * mu);
                double theta = 2 * 3.14159265358979323846 * rng_raw(&r);
                vv[(axis + 1) % 3] = _1mmu * cos(theta);
                vv[(axis + 2) % 3] = _1mmu * sin(theta);
                p.vx = vv[0] * c; p.vy = vv[1] * c; p.vz = vv[2] * c;
                p.w = energyToProduce;
                p.w0 = p.w;
                p.t = dt * rng_raw(&r);
                p.cell = (uint32_t)i;
                p.x = loc.x; p.y = loc.y; p.z = loc.z;
                repair_outside(o, &p, mc, 1e-8);
                p.w0 = fabs(p.w);
                p.pid = (uint32_t)(pidBase + nE + fpk);
                p.draw = 0;
                o->st.energy_emitted += p.w;
                bank_push(&o->bank, &p);
            }
        }
    }
    o->st.emitted_faces = fHi - fLo;
    return 0;
}

/* The HandleAll loop (manager/MonteCarloManagerSerial.hpp:267-383): every
 * particle is stepped to census, escape or removal. */
int orc_phase_transport(Oracle *o) {
    memset(o->segs, 0, sizeof(uint64_t) * o->N);
    /* every pid of the step (over all shards) is below this */
    o->pidLimit = o->nCenGlobal + o->nCellEmitGlobal + o->nFaceEmitGlobal;
    if (!o->pidLimit) o->pidLimit = 1;
    const int sharded = o->shards > 1;
    double *tally = sharded ? o->dep : o->eint;   /* sharded: deposits are summed over the ranks first */
    if (sharded) memset(o->dep, 0, sizeof(double) * o->N);
    for (uint64_t q = 0; q < o->bank.n; ++q) {
        Part p = o->bank.p[q];
        Rng r;
        memset(&r, 0, sizeof(r));
        r.seed = o->d.seed; r.tag = TAG_TRANSPORT; r.step = o->step; r.pid = p.pid; r.draw = p.draw;
        uint64_t nseg = 0;
        for (;;) {
            if (++nseg > HISTORY_SEGMENT_CAP) { raise(o, STORM_DERR_HISTORY_CAP, p.cell, p.pid); break; }
            o->segs[p.cell]++;
            o->st.segments++;
            uint32_t cell = p.cell;
            StepOut so;
            physics_step(o, &p, &r, &so);
            if (so.error) { raise(o, so.error, cell, p.pid); break; }
            tally[cell] += so.dmat;
            o->eradAvg[cell] += so.derad;
            o->st.energy_deposited += so.dmat;
            if (so.usedRW) o->st.rw_steps++;
            int m = manager_handle(o, &p, &so);
            if (m == 0) continue;
            if (m == 1) {
                o->st.census_out_pre_comb++;
                o->st.energy_census_pre_comb += p.w;
                p.draw = r.draw;
                bank_push(&o->census, &p);
            } else if (m == 2) {
                o->st.cutoff++;
            } else if (m == 3) {
                o->st.escaped++;
                o->st.energy_escaped += p.w;
            } else {
                raise(o, STORM_DERR_NOT_ON_BOUNDARY, cell, p.pid);
            }
            break;
        }
        if (o->derr) return -1;
    }
    o->bank.n = 0;
    if (sharded) {   /* exchange 1: deposits and time-averaged radiation, per cell */
        const uint64_t N = o->N;
        double *buf = (double *)malloc(sizeof(double) * 2 * (N ? N : 1));
        memcpy(buf, o->dep, sizeof(double) * N);
        memcpy(buf + N, o->eradAvg, sizeof(double) * N);
        int rc = exchange_sum(o, buf, 2 * N);
        for (uint64_t i = 0; i < N; ++i) o->eint[i] += buf[i];
        memcpy(o->eradAvg, buf + N, sizeof(double) * N);
        free(buf);
        if (rc) return -1;
    }
    return 0;
}

/* Deterministic reduction used by the engine for the comb's total weight:
 * partial sum t adds v[t], v[t + 1024], ... in order, then a pairwise tree. */
static double blocked_sum(const double *v, uint64_t n) {
    double part[1024];
    for (uint64_t t = 0; t < 1024; ++t) {
        double s = 0.0;
        for (uint64_t q = t; q < n; q += 1024) s += v[q];
        part[t] = s;
    }
    for (uint64_t w = 512; w >= 1; w >>= 1)
        for (uint64_t t = 0; t < w; ++t) part[t] = part[t] + part[t + w];
    return part[0];
}

typedef struct { uint64_t key; uint64_t idx; } KeyIdx;
static int cmp_key(const void *a, const void *b) {
    const KeyIdx *x = (const KeyIdx *)a, *y = (const KeyIdx *)b;
    return x->key < y->key ? -1 : (x->key > y->key ? 1 : 0);
}

/* CombPopulationControl::activate (population/CombPopulationControl.hpp:79-253).
 * Within a cell particles are ordered by the keyed bijection orc_comb_key
 * (the reference orders by id and std::shuffles with a function-static engine). */
static int orc_phase_comb_sharded(Oracle *o);

int orc_phase_comb(Oracle *o) {
    if (o->shards > 1) return orc_phase_comb_sharded(o);
    const uint64_t N = o->N;
    Bank in = o->census;
    Bank out = {NULL, 0, 0};
    uint64_t nz = 0;
    const int b = pid_bits(o->pidLimit);
    KeyIdx *ki = (KeyIdx *)malloc(sizeof(KeyIdx) * (in.n ? in.n : 1));
    for (uint64_t q = 0; q < in.n; ++q) {
        const Part *p = &in.p[q];
        if (outside_box(o, v3(p->x, p->y, p->z))) { raise(o, STORM_DERR_COMB_OUTSIDE, p->cell, p->pid); break; }
        if (!isfinite(p->w) || p->w < 0.0) { raise(o, STORM_DERR_COMB_WEIGHT, p->cell, p->pid); break; }
        if (p->w == 0.0) continue;
        ki[nz].key = ((uint64_t)p->cell << b) | orc_comb_key(o->d.seed, o->step, p->pid, b);
        ki[nz].idx = q;
        ++nz;
    }
    if (o->derr) { free(ki); return -1; }
    qsort(ki, nz, sizeof(KeyIdx), cmp_key);
    uint64_t *start = (uint64_t *)calloc(N + 1, sizeof(uint64_t));
    for (uint64_t q = 0; q < nz; ++q) start[(ki[q].key >> b) + 1]++;
    for (uint64_t i = 0; i < N; ++i) start[i + 1] += start[i];
    double *W = (double *)calloc(N ? N : 1, sizeof(double));
    for (uint64_t i = 0; i < N; ++i) {
        double s = 0.0;
        for (uint64_t q = start[i]; q < start[i + 1]; ++q) s += in.p[ki[q].idx].w;
        W[i] = s;
    }
    double totalWeight = blocked_sum(W, N);
    if (!isfinite(totalWeight)) { raise(o, STORM_DERR_COMB_TOTAL, 0, 0); }
    if (o->derr || totalWeight == 0.0) {
        free(ki); free(start); free(W);
        o->census.n = 0;
        return o->derr ? -1 : 0;
    }
    uint64_t Ntotal = (uint64_t)((double)(N * o->d.comb_nmin) * o->d.comb_factor);
    const uint64_t Nmin = o->d.comb_nmin;
    for (uint64_t i = 0; i < N; ++i) {
        uint64_t cnt = start[i + 1] - start[i];
        uint64_t share = (uint64_t)((double)Ntotal * W[i] / totalWeight);
        uint64_t lo = share > Nmin ? share : Nmin;
        uint64_t NinCell = (Nmin * 20 < lo) ? Nmin * 20 : lo;
        V3 mc = center(o, i);
        if (cnt <= NinCell) {
            double weight_ideal = W[i] / (double)NinCell;
            for (uint64_t q = start[i]; q < start[i + 1]; ++q) {
                Part p = in.p[ki[q].idx];
                if (p.w > 2 * weight_ideal) {
                    uint64_t Nsplit = (uint64_t)ceil(p.w / weight_ideal);
                    double ws = p.w / (double)Nsplit;
                    p.w = ws; p.w0 = ws; p.cell = (uint32_t)i; p.t = 0;
                    for (uint64_t s = 0; s < Nsplit; ++s) bank_push(&out, &p);
                } else {
                    bank_push(&out, &p);
                }
            }
            continue;
        }
        double new_energy = W[i] / (double)NinCell;
        double r = orc_uniform(o->d.seed, TAG_COMB, o->step, (uint32_t)i, 0);
        uint64_t comb_index = 0;
        double cum = 0;
        for (uint64_t q = start[i]; q < start[i + 1]; ++q) {
            const Part *src = &in.p[ki[q].idx];
            while ((cum + src->w) > ((double)comb_index + r) * new_energy) {
                ++comb_index;
                Part p = *src;
                p.cell = (uint32_t)i; p.t = 0; p.w = new_energy; p.w0 = new_energy;
                bank_push(&out, &p);
            }
            cum += src->w;
        }
        (void)mc;
    }
    /* outside-box repair of the result (:228-250) */
    for (uint64_t q = 0; q < out.n; ++q) {
        Part *p = &out.p[q];
        V3 loc = v3(p->x, p->y, p->z);
        if (!outside_box(o, loc)) continue;
        V3 mc = center(o, p->cell), original = loc, direction = vsub(mc, original);
        double t = 1e-6;
        while (outside_box(o, loc) && t < 1.0) { loc = vadd(original, vscale(t, direction)); t *= 2; }
        if (outside_box(o, loc)) loc = mc;
        p->x = loc.x; p->y = loc.y; p->z = loc.z;
    }
    for (uint64_t q = 0; q < out.n; ++q) { out.p[q].id = q; out.p[q].pid = (uint32_t)q; }
    free(ki); free(start); free(W);
    free(o->census.p);
    o->census = out;
    o->st.census_out = out.n;
    for (uint64_t q = 0; q < out.n; ++q) o->st.energy_census_out += out.p[q].w;
    return 0;
}

/* #{k >= 0 : (k + r) E < P}: the comb index a sequential walk holds once it
 * has passed weight P (the loop condition of :203-222 with cum = P). */
static uint64_t teeth_below(double P, double r, double E) {
    if (!(P > 0.0)) return 0;
    double g = P / E - r;
    uint64_t k = g > 0.0 ? (uint64_t)ceil(g) : 0;
    while (k > 0 && ((double)(k - 1) + r) * E >= P) --k;
    while (((double)k + r) * E < P) ++k;
    return k;
}

/* CombPopulationControl::activate over particle shards.  The census is sorted
 * by (shard, cell, keyed hash of pid); each (shard, cell) run's weight and
 * count are summed locally and exchanged, so that every rank sees every run.
 * A cell's targets come from its global weight (the shards' run weights added
 * in shard order) and count.  A combed cell's teeth are placed along the
 * cell's runs in shard order: run s starts at the weight P of the runs below it
 * and at the comb index teeth_below(P).  The new census stays with its shard,
 * in (shard, cell) order; exchange 3 gives every rank the shards' census
 * counts and the census energy per cell. */
static int orc_phase_comb_sharded(Oracle *o) {
    const uint64_t N = o->N;
    const uint32_t S = o->shards;
    const uint64_t R = (uint64_t)S * N;
    Bank in = o->census;
    Bank out = {NULL, 0, 0};
    uint64_t nz = 0;
    const int b = pid_bits(o->pidLimit);
    KeyIdx *ki = (KeyIdx *)malloc(sizeof(KeyIdx) * (in.n ? in.n : 1));
    for (uint64_t q = 0; q < in.n; ++q) {
        const Part *p = &in.p[q];
        if (outside_box(o, v3(p->x, p->y, p->z))) { raise(o, STORM_DERR_COMB_OUTSIDE, p->cell, p->pid); break; }
        if (!isfinite(p->w) || p->w < 0.0) { raise(o, STORM_DERR_COMB_WEIGHT, p->cell, p->pid); break; }
        if (p->w == 0.0) continue;
        const uint64_t run = (uint64_t)shard_of_pid(o, p->pid) * N + p->cell;
        ki[nz].key = (run << b) | orc_comb_key(o->d.seed, o->step, p->pid, b);
        ki[nz].idx = q;
        ++nz;
    }
    if (o->derr) { free(ki); return -1; }
    qsort(ki, nz, sizeof(KeyIdx), cmp_key);
    uint64_t *start = (uint64_t *)calloc(R + 1, sizeof(uint64_t));
    for (uint64_t q = 0; q < nz; ++q) start[(ki[q].key >> b) + 1]++;
    for (uint64_t r = 0; r < R; ++r) start[r + 1] += start[r];
    /* exchange 2: run weights and counts */
    double *WC = (double *)calloc(2 * R, sizeof(double));
    for (uint64_t r = 0; r < R; ++r) {
        double s = 0.0;
        for (uint64_t q = start[r]; q < start[r + 1]; ++q) s += in.p[ki[q].idx].w;
        WC[r] = s;
        WC[R + r] = (double)(start[r + 1] - start[r]);
    }
    int rc = exchange_sum(o, WC, 2 * R);
    double *Wc = (double *)calloc(N ? N : 1, sizeof(double));
    uint64_t *cnt = (uint64_t *)calloc(N ? N : 1, sizeof(uint64_t));
    for (uint64_t c = 0; c < N; ++c) {
        double w = 0.0;
        uint64_t k = 0;
        for (uint32_t s = 0; s < S; ++s) { w += WC[(uint64_t)s * N + c]; k += (uint64_t)WC[R + (uint64_t)s * N + c]; }
        Wc[c] = w;
        cnt[c] = k;
    }
    double totalWeight = blocked_sum(Wc, N);
    if (!isfinite(totalWeight)) raise(o, STORM_DERR_COMB_TOTAL, 0, 0);
    double *xc = (double *)calloc(S + N, sizeof(double));   /* exchange 3: shard census counts | census energy */
    if (!rc && !o->derr && totalWeight != 0.0) {
        uint64_t Ntotal = (uint64_t)((double)(N * o->d.comb_nmin) * o->d.comb_factor);
        const uint64_t Nmin = o->d.comb_nmin;
        for (uint32_t s = o->shardLo; s < o->shardHi; ++s) {
            for (uint64_t c = 0; c < N; ++c) {
                const uint64_t r0 = start[(uint64_t)s * N + c], r1 = start[(uint64_t)s * N + c + 1];
                if (r0 == r1) continue;
                const uint64_t before = out.n;
                uint64_t share = (uint64_t)((double)Ntotal * Wc[c] / totalWeight);
                uint64_t lo = share > Nmin ? share : Nmin;
                uint64_t NinCell = (Nmin * 20 < lo) ? Nmin * 20 : lo;
                if (cnt[c] <= NinCell) {
                    double weight_ideal = Wc[c] / (double)NinCell;
                    for (uint64_t q = r0; q < r1; ++q) {
                        Part p = in.p[ki[q].idx];
                        if (p.w > 2 * weight_ideal) {
                            uint64_t Nsplit = (uint64_t)ceil(p.w / weight_ideal);
                            double ws = p.w / (double)Nsplit;
                            p.w = ws; p.w0 = ws; p.cell = (uint32_t)c; p.t = 0;
                            for (uint64_t k = 0; k < Nsplit; ++k) { bank_push(&out, &p); xc[S + c] += ws; }
                        } else {
                            bank_push(&out, &p);
                            xc[S + c] += p.w;
                        }
                    }
                } else {
                    double new_energy = Wc[c] / (double)NinCell;
                    double r = orc_uniform(o->d.seed, TAG_COMB, o->step, (uint32_t)c, 0);
                    double cum = 0.0;
                    for (uint32_t t = 0; t < s; ++t) cum += WC[(uint64_t)t * N + c];
                    uint64_t comb_index = teeth_below(cum, r, new_energy);
                    for (uint64_t q = r0; q < r1; ++q) {
                        const Part *src = &in.p[ki[q].idx];
                        while ((cum + src->w) > ((double)comb_index + r) * new_energy) {
                            ++comb_index;
                            Part p = *src;
                            p.cell = (uint32_t)c; p.t = 0; p.w = new_energy; p.w0 = new_energy;
                            bank_push(&out, &p);
                            xc[S + c] += new_energy;
                        }
                        cum += src->w;
                    }
                }
                xc[s] += (double)(out.n - before);
            }
        }
    }
    if (!rc && exchange_sum(o, xc, S + N)) rc = -1;
    for (uint32_t s = 0; s < S; ++s) o->shardCensus[s] = (uint64_t)xc[s];
    for (uint64_t c = 0; c < N; ++c) o->eradCensus[c] = xc[S + c];
    /* outside-box repair of the result (:228-250) */
    for (uint64_t q = 0; q < out.n; ++q) {
        Part *p = &out.p[q];
        V3 loc = v3(p->x, p->y, p->z);
        if (!outside_box(o, loc)) continue;
        V3 mc = center(o, p->cell), original = loc, direction = vsub(mc, original);
        double t = 1e-6;
        while (outside_box(o, loc) && t < 1.0) { loc = vadd(original, vscale(t, direction)); t *= 2; }
        if (outside_box(o, loc)) loc = mc;
        p->x = loc.x; p->y = loc.y; p->z = loc.z;
    }
    const uint64_t pid0 = census_offset(o, o->shardLo);
    for (uint64_t q = 0; q < out.n; ++q) { out.p[q].id = pid0 + q; out.p[q].pid = (uint32_t)(pid0 + q); }
    free(ki); free(start); free(WC); free(Wc); free(cnt); free(xc);
    free(o->census.p);
    o->census = out;
    o->st.census_out = out.n;
    for (uint64_t q = 0; q < out.n; ++q) o->st.energy_census_out += out.p[q].w;
    return (rc || o->derr) ? -1 : 0;
}

/* RadiationIMC::postStep (radiation/RadiationIMC.hpp:1887-2029), gray, no hydro. */
int orc_phase_poststep(Oracle *o, double dt) {
    const uint64_t N = o->N;
    for (uint64_t i = 0; i < N; ++i) o->eradAvg[i] /= (dt * o->vol[i]);
    if (!o->d.no_hydro_feedback) {
        for (uint64_t i = 0; i < N; ++i) {
            double E = o->eint[i];
            if (E < 0.0) {   /* throwIfNegativeInternalEnergy :771-817 */
                double thermalScale = o->d.arad * pow(o->T[i], 4) * o->vol[i];
                if (thermalScale < 1e-30) thermalScale = 1e-30;
                double ratio = fabs(E) / thermalScale;
                if (ratio < 0.1) o->eint[i] = o->ceint[i] > 0.0 ? o->ceint[i] : 0.0;
                else raise(o, STORM_DERR_NEGATIVE_ENERGY, i, 0);
            }
            /* synchronizeMaterialCell :830-866 */
            double spec = o->eint[i] / o->mass[i];
            o->ceint[i] = o->eint[i];
            o->T[i] = eos_T(o, o->mass[i] / o->vol[i], spec);
        }
    }
    if (o->shards == 1) {   /* sharded: the comb's exchange filled it */
        for (uint64_t i = 0; i < N; ++i) o->eradCensus[i] = 0.0;
        for (uint64_t q = 0; q < o->census.n; ++q) o->eradCensus[o->census.p[q].cell] += o->census.p[q].w;
    }
    o->step++;
    return o->derr ? -1 : 0;
}

int orc_phase_stats(Oracle *o, StormStepStats *s) {
    *s = o->st;
    return 0;
}

int orc_step(Oracle *o, double dt, StormStepStats *stats) {
    int rc = orc_phase_begin(o, dt);
    if (!rc) rc = orc_phase_prestep(o, dt);
    if (!rc) rc = orc_phase_emit(o, dt);
    if (!rc) rc = orc_phase_transport(o);
    if (!rc && o->d.comb_enabled) rc = orc_phase_comb(o);
    if (!rc && !o->d.comb_enabled) {
        for (uint64_t q = 0; q < o->census.n; ++q) o->census.p[q].pid = (uint32_t)q;
        o->st.census_out = o->census.n;
    }
    if (!rc) rc = orc_phase_poststep(o, dt);
    if (stats) *stats = o->st;
    return rc;
}

/* ------------------------------------------------------------------ state access */
static void put_soa(const Bank *b, StormParticlesSoA *out) {
    for (uint64_t q = 0; q < b->n && q < out->count; ++q) {
        const Part *p = &b->p[q];
        out->x[q] = p->x; out->y[q] = p->y; out->z[q] = p->z;
        out->vx[q] = p->vx; out->vy[q] = p->vy; out->vz[q] = p->vz;
        out->time_left[q] = p->t; out->weight[q] = p->w; out->initial_weight[q] = p->w0;
        out->cell[q] = p->cell;
        if (out->id) out->id[q] = p->pid;
    }
}
int orc_set_census(Oracle *o, const StormParticlesSoA *in) {
    o->census.n = 0;
    for (uint64_t q = 0; q < in->count; ++q) {
        Part p;
        memset(&p, 0, sizeof(p));
        p.x = in->x[q]; p.y = in->y[q]; p.z = in->z[q];
        p.vx = in->vx[q]; p.vy = in->vy[q]; p.vz = in->vz[q];
        p.t = in->time_left[q]; p.w = in->weight[q]; p.w0 = in->initial_weight[q];
        p.cell = in->cell[q];
        p.pid = (uint32_t)q;
        bank_push(&o->census, &p);
    }
    o->pidLimit = in->count ? in->count : 1;
    return 0;
}
uint64_t orc_census_count(Oracle *o) { return o->census.n; }
int orc_get_census(Oracle *o, StormParticlesSoA *out) { put_soa(&o->census, out); return 0; }
uint64_t orc_bank_count(Oracle *o) { return o->bank.n; }
int orc_get_bank(Oracle *o, StormParticlesSoA *out) { put_soa(&o->bank, out); return 0; }
int orc_get_cell_arrays(Oracle *o, double *T, double *eint, double *eradAvg, double *eradCensus, double *sigA,
                        double *fleck, uint64_t *segs) {
    for (uint64_t i = 0; i < o->N; ++i) {
        if (T) T[i] = o->T[i];
        if (eint) eint[i] = o->eint[i];
        if (eradAvg) eradAvg[i] = o->eradAvg[i];
        if (eradCensus) eradCensus[i] = o->eradCensus[i];
        if (sigA) sigA[i] = o->sigA[i];
        if (fleck) fleck[i] = o->fleck[i];
        if (segs) segs[i] = o->segs[i];
    }
    return 0;
}
int orc_set_cell_physics(Oracle *o, const double *sigA, const double *sigS, const double *fleck) {
    for (uint64_t i = 0; i < o->N; ++i) {
        if (sigA) o->sigA[i] = sigA[i];
        if (sigS) o->sigS[i] = sigS[i];
        if (fleck) o->fleck[i] = fleck[i];
        if (o->d.with_random_walk) {   /* precomputeRandomWalkData with the given tables */
            double sigmaT = o->sigA[i] + o->sigS[i];
            o->rwSigT[i] = sigmaT;
            uint32_t ii, jj, kk;
            cell_ijk(o, i, &ii, &jj, &kk);
            double dx = o->xe[ii + 1] - o->xe[ii], dy = o->ye[jj + 1] - o->ye[jj], dz = o->ze[kk + 1] - o->ze[kk];
            double ax = dy * dz, ay = dz * dx, az = dx * dy;
            double S = 0.0;
            S += ax; S += ax; S += ay; S += ay; S += az; S += az;
            double chord = (S > 0.0) ? 4.0 * o->vol[i] / S : 0.0;
            o->rwElig[i] = (sigmaT * chord >= o->d.rw_min_cell_optical_depth);
        }
    }
    return 0;
}
int orc_get_emission(Oracle *o, uint64_t *photons, double *energy) {
    for (uint64_t i = 0; i < o->N; ++i) {
        if (photons) photons[i] = o->photons[i];
        if (energy) energy[i] = o->emitE[i];
    }
    return 0;
}
int orc_set_face_temperature(Oracle *o, int face, double T) {
    if (face < 0 || face > 5) return -1;
    o->faces[face].source_temperature = T;
    return 0;
}
int orc_last_error(Oracle *o, int32_t *derr, uint64_t *cell, uint64_t *particle) {
    if (derr) *derr = o->derr;
    if (cell) *cell = o->derrCell;
    if (particle) *particle = o->derrParticle;
    return 0;
}
uint32_t orc_step_index(Oracle *o) { return o->step; }

/* One segment per replay item: RadiationIMC::step + the manager's handling. */
int orc_replay_segments(Oracle *o, StormReplayBatch *b) {
    for (uint64_t q = 0; q < b->n; ++q) {
        Part p;
        memset(&p, 0, sizeof(p));
        p.x = b->x[q]; p.y = b->y[q]; p.z = b->z[q];
        p.vx = b->vx[q]; p.vy = b->vy[q]; p.vz = b->vz[q];
        p.t = b->time_left[q]; p.w = b->weight[q]; p.w0 = b->initial_weight[q];
        p.cell = b->cell[q];
        Rng r;
        memset(&r, 0, sizeof(r));
        r.tape_mode = 1; r.tape = b->tape + b->tape_offset[q]; r.len = b->tape_length[q];
        StepOut so;
        physics_step(o, &p, &r, &so);
        b->phys_x[q] = p.x; b->phys_y[q] = p.y; b->phys_z[q] = p.z;
        b->phys_vx[q] = p.vx; b->phys_vy[q] = p.vy; b->phys_vz[q] = p.vz;
        b->phys_time_left[q] = p.t; b->phys_weight[q] = p.w;
        b->phys_status[q] = so.error ? -1 : so.status;
        b->phys_next_cell[q] = (so.status == CELL_MOVE) ? (uint32_t)so.next : UINT32_MAX;
        b->dep_material[q] = so.dmat;
        b->dep_erad[q] = so.derad;
        b->used_random_walk[q] = so.usedRW;
        b->draws_used[q] = r.pos;
        int m = so.error ? -1 : manager_handle(o, &p, &so);
        b->mgr_x[q] = p.x; b->mgr_y[q] = p.y; b->mgr_z[q] = p.z;
        b->mgr_vx[q] = p.vx; b->mgr_vy[q] = p.vy; b->mgr_vz[q] = p.vz;
        b->mgr_cell[q] = p.cell;
        b->mgr_status[q] = r.exhausted ? -2 : m;
    }
    return 0;
}
