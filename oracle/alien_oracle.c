/*
 * alien_oracle.c - CPU restatement of ALIEN's per-timestep physics stage.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the B200 engine:
 * only the tests, the package's smoke check and the benchmark's CPU-baseline
 * leg load it.  The engine never calls it and has no CPU fallback.
 *
 * One source, two builds (see oracle/Makefile):
 *   liboracle_f64.so   REAL=double, single thread: the parity oracle.
 *   liboracle_f32.so   REAL=float, OpenMP: the timed CPU baseline.
 *
 * It restates, step for step, _SimulationKernelsLauncher::calcTimestep
 * (source/EngineGpuKernels/SimulationKernelsLauncher.cu:25-91) for cells whose
 * cell function is inactive, under the deterministic definitions shared with
 * the engine (each is cited where it is applied):
 *   D1 snapshot semantics: the pair-force phase reads positions from before
 *      the phase; overlap pushes are summed and applied after it (the
 *      reference writes cell->pos in place, CellProcessor.cuh:276,306).
 *   D2 sums are exact-order-independent (engine: fixed-point integers).
 *   D3 random draws come from a counter-based hash of (object id, timestep,
 *      draw site) instead of the shared cursor of CudaNumberGenerator.cuh:99-103.
 *   D4 lock-based pair updates (SystemDoubleLock::tryLock) are replaced by
 *      fixed rules: a cell gains at most one new bond per step (mutual
 *      smallest-id choice); particle merges go into particles that are not
 *      merging themselves; inner friction is one Jacobi sweep with one
 *      pair-average per bond.
 *   D5 the slot map keeps cells in storage order; a scan sees the first 10
 *      cells of a slot (Map.cuh:117-125, CellProcessor.cuh:165); the particle
 *      map keeps the highest storage index ("last writer", Map.cuh:254).
 *   D6 new objects take ids in the order: radiation particles (by cell
 *      storage order), split particles (by particle order), particles from
 *      deleted cells (by cell order); objects are stored in ingest order with
 *      stable compaction.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/alien_b200.h"

#ifndef REAL
#define REAL double
#endif
typedef REAL real;

#define NEAR_ZERO ((real)1.0e-4f) /* Base/Definitions.h:27 */
#define MAX_BONDS 6
#define SLOT_SCAN_LEVELS 10 /* Map.cuh:117, CellProcessor.cuh:165 */

#if REAL_IS_FLOAT
#define R_SQRT sqrtf
#define R_ATAN2 atan2f
#define R_SIN sinf
#define R_COS cosf
#define R_REM remainderf
#define R_ABS fabsf
#define R_PI 3.1415926535897932384626433832795f
#else
#define R_SQRT sqrt
#define R_ATAN2 atan2
#define R_SIN sin
#define R_COS cos
#define R_REM remainder
#define R_ABS fabs
#define R_PI 3.1415926535897932384626433832795
#endif
#define RAD_TO_DEG ((real)180 / R_PI)
#define DEG_TO_RAD (R_PI / (real)180)

typedef struct {
    real x, y;
} vec2;

static inline vec2 v2(real x, real y) { vec2 r = {x, y}; return r; }
static inline vec2 vadd(vec2 a, vec2 b) { return v2(a.x + b.x, a.y + b.y); }
static inline vec2 vsub(vec2 a, vec2 b) { return v2(a.x - b.x, a.y - b.y); }
static inline vec2 vmul(vec2 a, real m) { return v2(a.x * m, a.y * m); }
static inline vec2 vdiv(vec2 a, real m) { return v2(a.x / m, a.y / m); }
static inline real vdot(vec2 a, vec2 b) { return a.x * b.x + a.y * b.y; }
static inline real vlen(vec2 a) { return R_SQRT(a.x * a.x + a.y * a.y); }
static inline real vlen2(vec2 a) { return a.x * a.x + a.y * a.y; }
static inline real rmax(real a, real b) { return a > b ? a : b; }
static inline real rmin(real a, real b) { return a < b ? a : b; }

/* Math::normalize, Math.cuh:246-255 */
static inline vec2 vnormalized(vec2 a)
{
    real l = vlen(a);
    if (l > NEAR_ZERO) return v2(a.x / l, a.y / l);
    return v2(1, 0);
}
/* Math::rotateQuarterClockwise / CounterClockwise, Math.cuh:157-169 */
static inline vec2 rotCW(vec2 a) { return v2(-a.y, a.x); }
static inline vec2 rotCCW(vec2 a) { return v2(a.y, -a.x); }

/* Math::angleOfVector, Math.cuh:140-155 (degrees clockwise from (0,-1)):
 * 90 - asin(-v.y/|v|) for v.x >= 0, asin(..) + 270 otherwise; both equal
 * 90 - atan2(-v.y, v.x) mod 360, the well-conditioned form used here */
static real angleOfVector(vec2 v)
{
    real l = vlen(v);
    if (l < NEAR_ZERO) return 0;
    real a = (real)90 - R_ATAN2(-v.y, v.x) * RAD_TO_DEG;
    return a < 0 ? a + (real)360 : a;
}
/* Math::unitVectorOfAngle, Math.cuh:134-138 */
static vec2 unitVectorOfAngle(real a)
{
    a *= DEG_TO_RAD;
    return v2(R_SIN(a), -R_COS(a));
}
/* Math::subtractAngle, Math.cuh:300-310 */
static real subtractAngle(real a, real b)
{
    real d = a - b;
    if (d > (real)360) d -= (real)360;
    if (d < (real)0) d += (real)360;
    return d;
}
/* Math::isAngleInBetween, Math.cuh:223-236 */
static int isAngleInBetween(real a1, real a2, real c)
{
    if (a1 == a2 && a1 != c) return 0;
    if (c < a1) {
        c += (real)360;
        a2 += (real)360;
    }
    if (a2 < c) a2 += (real)360;
    return a2 - a1 < (real)360;
}
/* Math::crossing, Math.cuh:363-395 */
static int crossing(vec2 s, vec2 e, vec2 os, vec2 oe)
{
    if ((s.x == os.x && s.y == os.y) || (s.x == oe.x && s.y == oe.y) || (e.x == os.x && e.y == os.y)
        || (e.x == oe.x && e.y == oe.y))
        return 0;
    vec2 p1 = s, v1 = vsub(e, s), p2 = os, vv2 = vsub(oe, os);
    real divisor = vv2.x * v1.y - vv2.y * v1.x;
    if (R_ABS(divisor) < NEAR_ZERO) return 0;
    real mue = (v1.x * (p2.y - p1.y) - v1.y * (p2.x - p1.x)) / divisor;
    if (mue < -NEAR_ZERO || mue > 1 + NEAR_ZERO) return 0;
    real lambda;
    if (R_ABS(v1.x) > NEAR_ZERO)
        lambda = (p2.x - p1.x + mue * vv2.x) / v1.x;
    else if (R_ABS(v1.y) > NEAR_ZERO)
        lambda = (p2.y - p1.y + mue * vv2.y) / v1.y;
    else
        return 0;
    return lambda >= NEAR_ZERO && lambda <= 1 - NEAR_ZERO;
}

/* floorInt, Base.cuh:83-90 */
static inline int floorInt(real v)
{
    int r = (int)v;
    if (r > v) --r;
    return r;
}

/* counter-based draw (D3): SplitMix64 finaliser (Steele, Lea & Flood,
 * "Fast splittable pseudorandom number generators", OOPSLA 2014) applied to
 * (timestep, site) and then to the object id; 24 high bits -> [0, 1). */
static inline uint64_t splitmix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static inline float draw(uint64_t id, uint64_t step, uint32_t site)
{
    uint64_t h = splitmix64(splitmix64(step ^ ((uint64_t)site << 56)) ^ id);
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}
enum { SITE_FORCE_DECAY = 1, SITE_RADIATION = 2, SITE_RADIATION_ENERGY = 3, SITE_RADIATION_ANGLE = 4,
       SITE_DEATH = 5, SITE_SPLIT = 6, SITE_SPLIT_ANGLE = 7 };

/* calcKernel / calcKernel_d, CellProcessor.cuh:92-119 */
static real sphKernel(real q)
{
    real r;
    if (q < 1)
        r = (real)2 / (real)3 - q * q + (real)0.5 * q * q * q;
    else if (q < 2) {
        r = (real)2 - q;
        r = r * r * r / 6;
    } else
        r = 0;
    return r * ((real)3 / ((real)2 * R_PI));
}
static real sphKernelD(real q)
{
    real r;
    if (q < 1)
        r = -2 * q + (real)3 / (real)2 * q * q;
    else if (q < 2)
        r = (real)-0.5 * ((real)2 - q) * ((real)2 - q);
    else
        r = 0;
    return r * ((real)3 / ((real)2 * R_PI));
}

typedef struct OracleWorld {
    int W, H;
    AlienPhysicsParams p;
    uint64_t timestep;
    uint64_t nextId;

    int64_t nCells, capCells;
    uint64_t* id;
    vec2 *pos, *vel;
    real *energy, *stiffness, *density;
    uint8_t *color, *maxConn, *numConn, *barrier, *alive;
    int32_t* livingState;
    uint32_t *age, *activationTime, *creatureId;
    int32_t* cellFunction;
    int32_t (*bond)[MAX_BONDS];
    real (*bondDist)[MAX_BONDS];
    real (*bondAngle)[MAX_BONDS];
    AlienCellTO* cold; /* ingest copy: fields the physics stage never changes */

    int64_t nParts, capParts;
    uint64_t* pid;
    vec2 *ppos, *pvel;
    real* penergy;
    uint8_t *pcolor, *pselected, *palive;
    uint64_t* plastAbsorbed; /* cell id, UINT64_MAX = none */

    uint64_t nAux;
    uint8_t* aux;

    /* per-step scratch */
    vec2 *posPrime, *force, *forceOld, *angleAcc;
    real *densNew, *energyAdd;
    int32_t *best, *newPartner;
    uint8_t *delAll, *delCell, *detachFlag, *setDying, *newlyDying;
    int32_t *slotHead, *slotNext, *slotRank, *slotOf; /* cell map */
    int32_t* pmap;                                    /* particle map, W*H */
    int32_t* ptarget;
    int32_t* pslot;
    uint8_t* pincoming;
    real *mergeE, *mergeMx, *mergeMy;
    uint64_t neuronActivity[ALIEN_B200_MAX_COLORS]; /* neuron cells that ran (statistics) */
    double externalEnergy;   /* the external energy pool */
    double backflowSum;      /* this step's backflow into the pool */
    uint64_t activeSources;  /* radiation sources active in this step (bit i: source i) */
} OracleWorld;

#define XALLOC(ptr, n) ((ptr) = calloc((size_t)((n) > 0 ? (n) : 1), sizeof(*(ptr))))

static void freeCells(OracleWorld* w)
{
    free(w->id); free(w->pos); free(w->vel); free(w->energy); free(w->stiffness); free(w->density);
    free(w->color); free(w->maxConn); free(w->numConn); free(w->barrier); free(w->alive);
    free(w->livingState); free(w->age); free(w->activationTime); free(w->creatureId); free(w->cellFunction);
    free(w->bond); free(w->bondDist); free(w->bondAngle); free(w->cold);
    free(w->posPrime); free(w->force); free(w->forceOld); free(w->angleAcc); free(w->densNew); free(w->energyAdd);
    free(w->best); free(w->newPartner); free(w->delAll); free(w->delCell); free(w->detachFlag);
    free(w->setDying); free(w->newlyDying); free(w->slotNext); free(w->slotRank); free(w->slotOf);
}
static void allocCells(OracleWorld* w, int64_t cap)
{
    w->capCells = cap;
    XALLOC(w->id, cap); XALLOC(w->pos, cap); XALLOC(w->vel, cap); XALLOC(w->energy, cap);
    XALLOC(w->stiffness, cap); XALLOC(w->density, cap); XALLOC(w->color, cap); XALLOC(w->maxConn, cap);
    XALLOC(w->numConn, cap); XALLOC(w->barrier, cap); XALLOC(w->alive, cap); XALLOC(w->livingState, cap);
    XALLOC(w->age, cap); XALLOC(w->activationTime, cap); XALLOC(w->creatureId, cap);
    XALLOC(w->cellFunction, cap); XALLOC(w->bond, cap); XALLOC(w->bondDist, cap); XALLOC(w->bondAngle, cap);
    XALLOC(w->cold, cap); XALLOC(w->posPrime, cap); XALLOC(w->force, cap); XALLOC(w->forceOld, cap);
    XALLOC(w->angleAcc, cap); XALLOC(w->densNew, cap); XALLOC(w->energyAdd, cap); XALLOC(w->best, cap);
    XALLOC(w->newPartner, cap); XALLOC(w->delAll, cap); XALLOC(w->delCell, cap); XALLOC(w->detachFlag, cap);
    XALLOC(w->setDying, cap); XALLOC(w->newlyDying, cap); XALLOC(w->slotNext, cap); XALLOC(w->slotRank, cap);
    XALLOC(w->slotOf, cap);
}
static void freeParts(OracleWorld* w)
{
    free(w->pid); free(w->ppos); free(w->pvel); free(w->penergy); free(w->pcolor); free(w->pselected);
    free(w->palive); free(w->plastAbsorbed); free(w->ptarget); free(w->pslot); free(w->pincoming); free(w->mergeE);
    free(w->mergeMx); free(w->mergeMy);
}
static void growParts(OracleWorld* w, int64_t cap)
{
    if (cap <= w->capParts) return;
#define GROW(ptr) ptr = realloc(ptr, sizeof(*(ptr)) * (size_t)cap)
    GROW(w->pid); GROW(w->ppos); GROW(w->pvel); GROW(w->penergy); GROW(w->pcolor); GROW(w->pselected);
    GROW(w->palive); GROW(w->plastAbsorbed); GROW(w->ptarget); GROW(w->pslot); GROW(w->pincoming); GROW(w->mergeE);
    GROW(w->mergeMx); GROW(w->mergeMy);
#undef GROW
    w->capParts = cap;
}

OracleWorld* oracle_create(int worldSizeX, int worldSizeY, const AlienPhysicsParams* params, uint64_t timestep)
{
    if (worldSizeX <= 0 || worldSizeY <= 0 || !params) return NULL;
    OracleWorld* w = calloc(1, sizeof(OracleWorld));
    w->W = worldSizeX;
    w->H = worldSizeY;
    w->p = *params;
    w->timestep = timestep;
    w->externalEnergy = params->externalEnergy;
    w->nextId = 1;
    allocCells(w, 1);
    growParts(w, 16);
    w->slotHead = malloc(sizeof(int32_t) * (size_t)w->W * (size_t)w->H);
    w->pmap = malloc(sizeof(int32_t) * (size_t)w->W * (size_t)w->H);
    for (int64_t s = 0; s < (int64_t)w->W * w->H; ++s) {
        w->slotHead[s] = -1;
        w->pmap[s] = -1;
    }
    return w;
}

void oracle_destroy(OracleWorld* w)
{
    if (!w) return;
    freeCells(w);
    freeParts(w);
    free(w->slotHead);
    free(w->pmap);
    free(w->aux);
    free(w);
}

void oracle_set_parameters(OracleWorld* w, const AlienPhysicsParams* params)
{
    w->p = *params;
    w->externalEnergy = params->externalEnergy;
    /* prepareForSimulationParametersChanges -> resetDensity,
     * SimulationKernelsLauncher.cu:93-97, CellProcessor.cuh:860-870 */
    for (int64_t i = 0; i < w->nCells; ++i) w->density[i] = 1;
}

uint64_t oracle_timestep(OracleWorld* w) { return w->timestep; }

/* BaseMap::correctPosition (int and float forms), Map.cuh:15-26 */
static inline int wrapInt(int v, int size) { return ((v % size) + size) % size; }
static inline vec2 correctPosition(const OracleWorld* w, vec2 p)
{
    int ix = floorInt(p.x), iy = floorInt(p.y);
    real fx = p.x - (real)ix, fy = p.y - (real)iy;
    ix = wrapInt(ix, w->W);
    iy = wrapInt(iy, w->H);
    return v2((real)ix + fx, (real)iy + fy);
}
/* BaseMap::correctDirection, Map.cuh:35-39 */
static inline vec2 correctDirection(const OracleWorld* w, vec2 d)
{
    return v2(R_REM(d.x, (real)w->W), R_REM(d.y, (real)w->H));
}
static inline int slotOfPos(const OracleWorld* w, vec2 p)
{
    int ix = wrapInt(floorInt(p.x), w->W), iy = wrapInt(floorInt(p.y), w->H);
    return ix + iy * w->W;
}

/* ---- ingest / egress: cudaCreateDataFromTO (DataAccessKernels.cu:363-387),
 *      ObjectFactory::createCellFromTO / createParticleFromTO
 *      (ObjectFactory.cuh:46-86), createCellTO (DataAccessKernels.cu:18-110) */
int oracle_set_data(OracleWorld* w, const AlienDataTO* to)
{
    int64_t nc = (int64_t)*to->numCells, np = (int64_t)*to->numParticles;
    freeCells(w);
    allocCells(w, nc > 0 ? nc : 1);
    w->nCells = nc;
    w->nextId = 1;
    for (int64_t i = 0; i < nc; ++i) {
        const AlienCellTO* c = &to->cells[i];
        w->cold[i] = *c;
        w->id[i] = c->id;
        w->pos[i] = correctPosition(w, v2(c->pos.x, c->pos.y));
        w->vel[i] = v2(c->vel.x, c->vel.y);
        w->energy[i] = c->energy;
        w->stiffness[i] = c->stiffness;
        w->density[i] = 1;
        w->color[i] = c->color;
        w->maxConn[i] = c->maxConnections;
        w->numConn[i] = c->numConnections;
        w->barrier[i] = c->barrier;
        w->alive[i] = 1;
        w->livingState[i] = c->livingState;
        w->age[i] = c->age;
        w->activationTime[i] = c->activationTime;
        w->creatureId[i] = c->creatureId;
        w->cellFunction[i] = c->cellFunction;
        for (int k = 0; k < MAX_BONDS; ++k) {
            w->bond[i][k] = k < c->numConnections ? c->connections[k].cellIndex : -1;
            w->bondDist[i][k] = c->connections[k].distance;
            w->bondAngle[i][k] = c->connections[k].angleFromPrevious;
        }
        if (c->id + 1 > w->nextId) w->nextId = c->id + 1;
    }
    w->nParts = 0;
    growParts(w, np + 16);
    for (int64_t i = 0; i < np; ++i) {
        const AlienParticleTO* q = &to->particles[i];
        w->pid[i] = q->id;
        w->ppos[i] = correctPosition(w, v2(q->pos.x, q->pos.y));
        w->pvel[i] = v2(q->vel.x, q->vel.y);
        w->penergy[i] = q->energy;
        w->pcolor[i] = q->color;
        w->pselected[i] = 0;
        w->palive[i] = 1;
        w->plastAbsorbed[i] = UINT64_MAX;
        if (q->id + 1 > w->nextId) w->nextId = q->id + 1;
    }
    w->nParts = np;
    free(w->aux);
    w->nAux = *to->numAuxiliaryData;
    w->aux = malloc(w->nAux > 0 ? w->nAux : 1);
    if (w->nAux) memcpy(w->aux, to->auxiliaryData, w->nAux);
    return 0;
}

void oracle_get_counts(OracleWorld* w, uint64_t* numCells, uint64_t* numParticles, uint64_t* numAux)
{
    uint64_t c = 0, q = 0;
    for (int64_t i = 0; i < w->nCells; ++i) c += w->alive[i];
    for (int64_t i = 0; i < w->nParts; ++i) q += w->palive[i];
    *numCells = c;
    *numParticles = q;
    *numAux = w->nAux;
}

int oracle_get_data(OracleWorld* w, const AlienDataTO* to)
{
    int32_t* newIndex = malloc(sizeof(int32_t) * (size_t)(w->nCells > 0 ? w->nCells : 1));
    int64_t n = 0;
    for (int64_t i = 0; i < w->nCells; ++i) newIndex[i] = w->alive[i] ? (int32_t)n++ : -1;
    for (int64_t i = 0; i < w->nCells; ++i) {
        if (!w->alive[i]) continue;
        AlienCellTO* c = &to->cells[newIndex[i]];
        *c = w->cold[i];
        c->id = w->id[i];
        c->pos.x = (float)w->pos[i].x;
        c->pos.y = (float)w->pos[i].y;
        c->vel.x = (float)w->vel[i].x;
        c->vel.y = (float)w->vel[i].y;
        c->energy = (float)w->energy[i];
        c->stiffness = (float)w->stiffness[i];
        c->color = w->color[i];
        c->maxConnections = w->maxConn[i];
        c->numConnections = w->numConn[i];
        c->barrier = w->barrier[i];
        c->livingState = w->livingState[i];
        c->age = w->age[i];
        c->activationTime = w->activationTime[i];
        for (int k = 0; k < MAX_BONDS; ++k) {
            if (k < w->numConn[i]) {
                c->connections[k].cellIndex = newIndex[w->bond[i][k]];
                c->connections[k].distance = (float)w->bondDist[i][k];
                c->connections[k].angleFromPrevious = (float)w->bondAngle[i][k];
            } else {
                c->connections[k].cellIndex = 0;
                c->connections[k].distance = 0;
                c->connections[k].angleFromPrevious = 0;
            }
        }
    }
    int64_t m = 0;
    for (int64_t i = 0; i < w->nParts; ++i) {
        if (!w->palive[i]) continue;
        AlienParticleTO* q = &to->particles[m++];
        memset(q, 0, sizeof(*q));
        q->id = w->pid[i];
        q->energy = (float)w->penergy[i];
        q->pos.x = (float)w->ppos[i].x;
        q->pos.y = (float)w->ppos[i].y;
        q->vel.x = (float)w->pvel[i].x;
        q->vel.y = (float)w->pvel[i].y;
        q->color = w->pcolor[i];
        q->selected = w->pselected[i];
    }
    *to->numCells = (uint64_t)n;
    *to->numParticles = (uint64_t)m;
    *to->numAuxiliaryData = w->nAux;
    if (w->nAux) memcpy(to->auxiliaryData, w->aux, w->nAux);
    free(newIndex);
    return 0;
}

/* ---- zones: SpotCalculator (SpotCalculator.cuh:12-251).  A parameter
 *      blends from its base value into the values of the zones that
 *      activate it, by each zone's weight at the position (0 in the core,
 *      rising to 1 over the fade-out radius + 1):
 *      base * prod(w_i) + sum_i v_i (1 - w_i) / (sum_i (1 - w_i) + prod(w_i)). */
enum { ZF_FRICTION, ZF_RIGIDITY, ZF_RADIATION_ABSORPTION, ZF_RADIATION_CELL_AGE_STRENGTH, ZF_CELL_MAX_FORCE,
       ZF_CELL_MIN_ENERGY, ZF_CELL_DEATH_PROBABILITY, ZF_CELL_FUSION_VELOCITY, ZF_CELL_MAX_BINDING_ENERGY,
       ZF_RADIATION_DISABLE_SOURCES };

static int zoneActivated(const AlienZone* z, int f)
{
    switch (f) {
    case ZF_FRICTION: return z->frictionActivated;
    case ZF_RIGIDITY: return z->rigidityActivated;
    case ZF_RADIATION_ABSORPTION: return z->radiationAbsorptionActivated;
    case ZF_RADIATION_CELL_AGE_STRENGTH: return z->radiationCellAgeStrengthActivated;
    case ZF_CELL_MAX_FORCE: return z->cellMaxForceActivated;
    case ZF_CELL_MIN_ENERGY: return z->cellMinEnergyActivated;
    case ZF_CELL_DEATH_PROBABILITY: return z->cellDeathProbabilityActivated;
    case ZF_CELL_FUSION_VELOCITY: return z->cellFusionVelocityActivated;
    case ZF_CELL_MAX_BINDING_ENERGY: return z->cellMaxBindingEnergyActivated;
    default: return z->radiationDisableSourcesActivated;
    }
}
static real zoneValue(const AlienZone* z, int f, int color)
{
    switch (f) {
    case ZF_FRICTION: return z->friction;
    case ZF_RIGIDITY: return z->rigidity;
    case ZF_RADIATION_ABSORPTION: return z->radiationAbsorption[color];
    case ZF_RADIATION_CELL_AGE_STRENGTH: return z->radiationCellAgeStrength[color];
    case ZF_CELL_MAX_FORCE: return z->cellMaxForce[color];
    case ZF_CELL_MIN_ENERGY: return z->cellMinEnergy[color];
    case ZF_CELL_DEATH_PROBABILITY: return z->cellDeathProbability[color];
    case ZF_CELL_FUSION_VELOCITY: return z->cellFusionVelocity;
    case ZF_CELL_MAX_BINDING_ENERGY: return z->cellMaxBindingEnergy;
    default: return z->radiationDisableSources ? 1 : 0;
    }
}
/* SpotCalculator::calcWeight, :183-210; delta = zone - position */
static real zoneWeight(const AlienZone* z, vec2 delta)
{
    if (z->shapeType == ALIEN_B200_SHAPE_RECTANGULAR) {
        real hw = (real)z->width / 2, hh = (real)z->height / 2;
        if (R_ABS(delta.x) > hw || R_ABS(delta.y) > hh) {
            vec2 d = v2(rmax(0, R_ABS(delta.x) - hw), rmax(0, R_ABS(delta.y) - hh));
            return rmin(1, vlen(d) / ((real)z->fadeoutRadius + 1));
        }
        return 0;
    }
    real distance = vlen(delta);
    return distance < (real)z->coreRadius ? 0 : rmin(1, (distance - (real)z->coreRadius) / ((real)z->fadeoutRadius + 1));
}
static real zoneWeightAt(const OracleWorld* w, const AlienZone* z, vec2 pos)
{
    return zoneWeight(z, correctDirection(w, vsub(v2(z->posX, z->posY), pos)));
}
/* SpotCalculator::calcParameter, :78-160 */
static real zoneParam(const OracleWorld* w, int f, vec2 pos, real base, int color)
{
    const AlienPhysicsParams* p = &w->p;
    if (p->numZones <= 0) return base;
    real baseFactor = 1, sum = 0;
    for (int i = 0; i < p->numZones; ++i) {
        if (!zoneActivated(&p->zones[i], f)) continue;
        real wi = zoneWeightAt(w, &p->zones[i], pos);
        baseFactor *= wi;
        sum += 1 - wi;
    }
    sum += baseFactor;
    real result = base * baseFactor;
    for (int i = 0; i < p->numZones; ++i) {
        if (!zoneActivated(&p->zones[i], f)) continue;
        real wi = zoneWeightAt(w, &p->zones[i], pos);
        result += zoneValue(&p->zones[i], f, color) * (1 - wi) / sum;
    }
    return result;
}
/* FlowFieldKernels.cu:10-44 */
static real flowHeight(const OracleWorld* w, const AlienZone* z, vec2 pos)
{
    real h = R_SQRT(vlen(correctDirection(w, vsub(pos, v2(z->posX, z->posY))))) * (real)z->flowStrength;
    return z->flowOrientation == 0 ? h : -h;
}
static vec2 zoneFlow(const OracleWorld* w, const AlienZone* z, vec2 pos)
{
    if (z->flowType == ALIEN_B200_FLOW_RADIAL) {
        real b = flowHeight(w, z, pos), down = flowHeight(w, z, vadd(pos, v2(0, 1))), right = flowHeight(w, z, vadd(pos, v2(1, 0)));
        vec2 r = v2(right - b, down - b);
        real a = ((real)90 + (real)z->flowDriftAngle) * DEG_TO_RAD; /* Math::rotateClockwise */
        return v2(r.x * R_COS(a) - r.y * R_SIN(a), r.x * R_SIN(a) + r.y * R_COS(a));
    }
    if (z->flowType == ALIEN_B200_FLOW_CENTRAL) {
        vec2 c = correctDirection(w, vsub(v2(z->posX, z->posY), pos));
        return vmul(c, (real)z->flowStrength / (vlen2(c) + 50));
    }
    if (z->flowType == ALIEN_B200_FLOW_LINEAR) return vmul(unitVectorOfAngle(z->flowAngle), (real)z->flowStrength);
    return v2(0, 0);
}
/* cudaApplyFlowFieldSettings with calcResultingFlowField (FlowFieldKernels.cu:48-89, SpotCalculator.cuh:58-78) */
static vec2 flowAcceleration(const OracleWorld* w, vec2 pos)
{
    const AlienPhysicsParams* p = &w->p;
    real baseFactor = 1, sum = 0;
    int any = 0;
    for (int i = 0; i < p->numZones; ++i) {
        if (p->zones[i].flowType == ALIEN_B200_FLOW_NONE) continue;
        real wi = zoneWeightAt(w, &p->zones[i], pos);
        baseFactor *= wi;
        sum += 1 - wi;
        any = 1;
    }
    if (!any) return v2(0, 0);
    sum += baseFactor;
    vec2 result = v2(0, 0);
    for (int i = 0; i < p->numZones; ++i) {
        if (p->zones[i].flowType == ALIEN_B200_FLOW_NONE) continue;
        real wi = zoneWeightAt(w, &p->zones[i], pos);
        result = vadd(result, vdiv(vmul(zoneFlow(w, &p->zones[i], pos), 1 - wi), sum));
    }
    return result;
}
/* RadiationProcessor::calcActiveSources, RadiationProcessor.cuh:42-59 */
static uint64_t calcActiveSources(const OracleWorld* w)
{
    const AlienPhysicsParams* p = &w->p;
    uint64_t mask = 0;
    for (int i = 0; i < p->numRadiationSources; ++i) {
        const AlienRadiationSource* r = &p->radiationSources[i];
        real disabled = zoneParam(w, ZF_RADIATION_DISABLE_SOURCES, v2(r->posX, r->posY), p->radiationDisableSources ? 1 : 0, 0);
        if (!(disabled > (real)0.5)) mask |= 1ull << i;
    }
    return mask;
}
/* createEnergyParticle's placement at a radiation source
 * (RadiationProcessor.cuh:252-343); draw sites as in the engine: base + 0
 * source choice, base + 1 + 2k / base + 2 + 2k the k-th circular try,
 * base + 21 the speed, base + 22 / 23 the rectangular offset */
#define SITE_SOURCE_RADIATION 32
#define SITE_SOURCE_DELETED_CELL 64
static void placeAtSource(const OracleWorld* w, uint64_t id, uint64_t T, uint32_t site, vec2* pos, vec2* vel)
{
    const AlienPhysicsParams* p = &w->p;
    uint64_t mask = w->activeSources;
    if (!mask) return;
    real sumRatios = 0;
    for (int i = 0; i < p->numRadiationSources; ++i)
        if ((mask >> i) & 1ull) sumRatios += p->radiationSources[i].strength;
    if (!(sumRatios > 0)) return;
    real r = draw(id, T, site);
    sumRatios = 0;
    int index = -1;
    for (int i = 0; i < p->numRadiationSources; ++i) {
        if (!((mask >> i) & 1ull)) continue;
        sumRatios += p->radiationSources[i].strength;
        if (r <= sumRatios) {
            index = i;
            break;
        }
    }
    if (index < 0) return;
    const AlienRadiationSource* src = &p->radiationSources[index];
    *pos = v2(src->posX, src->posY);
    real speed = (real)0.5 + (real)0.5 * draw(id, T, site + 21);
    if (src->shapeType == ALIEN_B200_SHAPE_CIRCULAR) {
        real radius = rmax(1, src->radius);
        vec2 delta = v2(0, 0);
        for (int k = 0; k < 10; ++k) {
            delta.x = (real)draw(id, T, site + 1 + 2 * k) * radius * 2 - radius;
            delta.y = (real)draw(id, T, site + 2 + 2 * k) * radius * 2 - radius;
            if (vlen(delta) <= radius) break;
        }
        *pos = vadd(*pos, delta);
        *vel = src->useAngle ? vmul(unitVectorOfAngle(src->angle), speed) : vmul(vnormalized(delta), speed);
    } else {
        real wd = src->width, ht = src->height;
        vec2 delta = v2((real)draw(id, T, site + 22) * wd - wd / 2, (real)draw(id, T, site + 23) * ht - ht / 2);
        *pos = vadd(*pos, delta);
        if (src->useAngle) {
            *vel = vmul(unitVectorOfAngle(src->angle), speed);
        } else {
            real round = rmin(wd, ht) / 2;
            vec2 c1 = v2(-wd / 2, -ht / 2), c2 = v2(wd / 2, -ht / 2), c3 = v2(-wd / 2, ht / 2), c4 = v2(wd / 2, ht / 2);
#define LMAX(v) rmax(R_ABS((v).x), R_ABS((v).y))
            vec2 v;
            if (LMAX(vsub(c1, delta)) <= round) {
                v = vnormalized(vsub(delta, vadd(c1, v2(round, round))));
            } else if (LMAX(vsub(c2, delta)) <= round) {
                v = vnormalized(vsub(delta, vadd(c2, v2(-round, round))));
            } else if (LMAX(vsub(c3, delta)) <= round) {
                v = vnormalized(vsub(delta, vadd(c3, v2(round, -round))));
            } else if (LMAX(vsub(c4, delta)) <= round) {
                v = vnormalized(vsub(delta, vadd(c4, v2(-round, -round))));
            } else {
                real dx1 = wd / 2 + delta.x, dx2 = wd / 2 - delta.x, dy1 = ht / 2 + delta.y, dy2 = ht / 2 - delta.y;
                v = v2(0, 0);
                if (dx1 <= dy1 && dx1 <= dy2 && delta.x <= 0) v.x = -1;
                if (dy1 <= dx1 && dy1 <= dx2 && delta.y <= 0) v.y = -1;
                if (dx2 <= dy1 && dx2 <= dy2 && delta.x > 0) v.x = 1;
                if (dy2 <= dx1 && dy2 <= dx2 && delta.y > 0) v.y = 1;
            }
#undef LMAX
            *vel = vmul(v, speed);
        }
    }
}
/* the external-energy backflow (RadiationProcessor.cuh:345-354), accepted
 * when the pool at the start of the step plus the amount stays within the
 * limit; returns the particle's energy */
static real backflow(OracleWorld* w, int color, real energy)
{
    const AlienPhysicsParams* p = &w->p;
    if (!p->externalEnergyControl || !(p->externalEnergyBackflowFactor[color] > 0)) return energy;
    real factor = p->externalEnergyBackflowFactor[color];
    double add = (double)(energy * factor);
    if (w->externalEnergy + add > (double)p->externalEnergyBackflowLimit) return energy;
    w->backflowSum += add;
    return energy * (1 - factor);
}
/* SimulationParametersUpdateService.cu:52-78 */
static void moveOnTorus(const OracleWorld* w, float* x, float* y, float vx, float vy, float dt)
{
    real px = *x, py = *y;
    if (R_ABS(vx) > NEAR_ZERO) px += (real)vx * dt;
    if (R_ABS(vy) > NEAR_ZERO) py += (real)vy * dt;
    vec2 c = correctPosition(w, v2(px, py));
    *x = (float)c.x;
    *y = (float)c.y;
}

/* ---- particle creation: ObjectFactory::createParticle (ObjectFactory.cuh
 *      :242-256) for particles above NEAR_ZERO */
static void createParticle(OracleWorld* w, vec2 pos, vec2 vel, int color, real energy)
{
    pos = correctPosition(w, pos);
    if (!(energy > NEAR_ZERO)) return;
    if (w->nParts == w->capParts) growParts(w, w->capParts * 2 + 16);
    int64_t k = w->nParts++;
    w->pid[k] = w->nextId++;
    w->ppos[k] = correctPosition(w, pos);
    w->pvel[k] = vel;
    w->penergy[k] = energy;
    w->pcolor[k] = (uint8_t)color;
    w->pselected[k] = 0;
    w->palive[k] = 1;
    w->plastAbsorbed[k] = UINT64_MAX;
}

/* RadiationProcessor::createEnergyParticle (RadiationProcessor.cuh:248-364):
 * at an active radiation source if there is one, then the external-energy
 * backflow; draws keyed by the emitting cell's id */
static void createEnergyParticle(OracleWorld* w, vec2 pos, vec2 vel, int color, real energy, uint64_t id, uint32_t site)
{
    placeAtSource(w, id, w->timestep, site, &pos, &vel);
    pos = correctPosition(w, pos);
    real kept = backflow(w, color, energy);
    createParticle(w, pos, vel, color, kept);
}

static inline int isBonded(const OracleWorld* w, int64_t i, int64_t j)
{
    for (int k = 0; k < w->numConn[i]; ++k)
        if (w->bond[i][k] == j) return 1;
    return 0;
}

/* ---- cell map (D5): slot lists in storage order, CellMap::set_block
 *      Map.cuh:95-130 */
static void buildCellMap(OracleWorld* w)
{
    int64_t nSlots = (int64_t)w->W * w->H;
    (void)nSlots;
    for (int64_t i = w->nCells - 1; i >= 0; --i) {
        if (!w->alive[i]) continue;
        int s = slotOfPos(w, w->pos[i]);
        w->slotOf[i] = s;
        w->slotNext[i] = w->slotHead[s];
        w->slotHead[s] = (int32_t)i;
    }
    for (int64_t i = 0; i < w->nCells; ++i) {
        if (!w->alive[i]) continue;
        int s = w->slotOf[i];
        if (w->slotHead[s] != (int32_t)i) continue;
        int r = 0;
        for (int32_t c = (int32_t)i; c >= 0; c = w->slotNext[c]) w->slotRank[c] = r++;
    }
}
/* every cell of the step was inserted (all are alive at the step start);
 * cells deleted during the step must be cleared as well */
static void clearCellMap(OracleWorld* w)
{
    for (int64_t i = 0; i < w->nCells; ++i) w->slotHead[w->slotOf[i]] = -1;
}

/* ---- CellProcessor::radiation, CellProcessor.cuh:725-773 */
static void radiationPhase(OracleWorld* w, uint64_t T)
{
    const AlienPhysicsParams* p = &w->p;
    for (int64_t i = 0; i < w->nCells; ++i) {
        if (!w->alive[i] || w->barrier[i]) continue;
        if (!(draw(w->id[i], T, SITE_RADIATION) < p->radiationProb)) continue;
        int c = w->color[i] % ALIEN_B200_MAX_COLORS;
        real factor = 0;
        if (w->energy[i] > (real)p->highRadiationMinCellEnergy[c]) factor += (real)p->highRadiationFactor[c];
        if ((int64_t)w->age[i] > (int64_t)p->radiationMinCellAge[c])
            factor += zoneParam(w, ZF_RADIATION_CELL_AGE_STRENGTH, w->pos[i], p->radiationCellAgeStrength[c], c);
        if (!(factor > 0)) continue;
        real e = w->energy[i];
        real loss = e * factor;
        loss = loss / (real)p->radiationProb;
        loss = 2 * loss * (real)draw(w->id[i], T, SITE_RADIATION_ENERGY);
        if (e > 1) {
            vec2 pv = vadd(vmul(w->vel[i], (real)p->radiationVelocityMultiplier),
                           vmul(unitVectorOfAngle((real)draw(w->id[i], T, SITE_RADIATION_ANGLE) * 360),
                                (real)p->radiationVelocityPerturbation));
            vec2 pp = vsub(vadd(w->pos[i], vmul(vnormalized(pv), (real)1.5)), pv);
            pp = correctPosition(w, pp);
            if (loss > e - 1) loss = e - 1;
            createEnergyParticle(w, pp, pv, w->color[i], loss, w->id[i], SITE_SOURCE_RADIATION);
            w->energy[i] -= loss;
        }
    }
}

/* ---- fluid pair forces, CellProcessor.cuh:122-283 (D1, D2, D4, D5) */
static void fluidPhase(OracleWorld* w)
{
    const AlienPhysicsParams* p = &w->p;
    const real h = (real)p->smoothingLength;
    const real R = h * 2;
    const int radiusInt = (int)ceilf(p->smoothingLength * 2);
    const real minDist = (real)p->cellMinDistance;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < w->nCells; ++i) {
        if (!w->alive[i]) continue;
        vec2 pi = w->pos[i], vi = w->vel[i];
        /* zone values at the cell, CellProcessor.cuh:149-152 */
        const real fusionVelocity = zoneParam(w, ZF_CELL_FUSION_VELOCITY, pi, p->cellFusionVelocity, 0);
        const real maxBindingEnergy = zoneParam(w, ZF_CELL_MAX_BINDING_ENERGY, pi, p->cellMaxBindingEnergy, 0);
        real dens = 0;
        vec2 Fp = v2(0, 0), Fv = v2(0, 0), dx = v2(0, 0);
        int64_t bestBarrier = -1;
        real bestBarrierDist = 0;
        int32_t best = -1;
        uint64_t bestId = UINT64_MAX;
        int bx = floorInt(pi.x) - radiusInt, by = floorInt(pi.y) - radiusInt;
        int scan = radiusInt * 2 + 1;
        for (int t = 0; t < scan * scan; ++t) {
            int sx = wrapInt(bx + t % scan, w->W), sy = wrapInt(by + t / scan, w->H);
            int32_t j = w->slotHead[sx + sy * w->W];
            for (int level = 0; level < SLOT_SCAN_LEVELS && j >= 0; ++level, j = w->slotNext[j]) {
                vec2 pd = correctDirection(w, vsub(pi, w->pos[j]));
                real d = vlen(pd);
                if (w->barrier[j] && d <= R) {
                    if (bestBarrier < 0 || d < bestBarrierDist || (d == bestBarrierDist && j < bestBarrier)) {
                        bestBarrier = j;
                        bestBarrierDist = d;
                    }
                }
                if (!w->barrier[j] && d <= R) {
                    dens += sphKernel(d / h) / (h * h);
                    if (j != i) {
                        if (!w->barrier[i] && d < minDist) dx = vadd(dx, vmul(pd, minDist / 5));
                        if (!isBonded(w, i, j)) {
                            vec2 vd = vsub(vi, w->vel[j]);
                            real di = w->density[i], dj = w->density[j];
                            real factor = di / (di * di) + dj / (dj * dj);
                            if (R_ABS(d) > NEAR_ZERO) {
                                real kd = sphKernelD(d / h) / (h * h * h);
                                Fp = vadd(Fp, vmul(vdiv(pd, -d), factor * kd));
                                Fv = vadd(Fv, vmul(vdiv(vd, dj), d * kd / (d * d + (real)0.25)));
                            }
                            if (vlen(vd) >= fusionVelocity && w->numConn[i] < w->maxConn[i]
                                && w->numConn[j] < w->maxConn[j] && w->energy[i] <= maxBindingEnergy
                                && w->energy[j] <= maxBindingEnergy && !w->barrier[i] && !w->barrier[j]) {
                                if (w->id[j] < bestId) {
                                    bestId = w->id[j];
                                    best = j;
                                }
                            }
                        }
                    }
                }
            }
        }
        vec2 F = v2(0, 0);
        if (bestBarrier >= 0) {
            int64_t b = bestBarrier;
            vec2 r = v2(0, 0);
            if (w->numConn[b] <= 1) {
                r = correctDirection(w, vsub(pi, w->pos[b]));
            } else {
                real angleToCell = angleOfVector(correctDirection(w, vsub(pi, w->pos[b])));
                int n = w->numConn[b];
                for (int k = 0; k < n; ++k) {
                    int32_t c1 = w->bond[b][k], c2 = w->bond[b][(k + 1) % n];
                    real a1 = angleOfVector(correctDirection(w, vsub(w->pos[c1], w->pos[b])));
                    real a2 = angleOfVector(correctDirection(w, vsub(w->pos[c2], w->pos[b])));
                    if (isAngleInBetween(a1, a2, angleToCell)) {
                        r = rotCCW(vsub(w->pos[c2], w->pos[c1]));
                        break;
                    }
                }
            }
            vec2 vr = vsub(vi, w->vel[b]);
            real dvr = vdot(vr, r);
            if (dvr < 0) {
                real trr = rmax((real)0.05, vlen2(r));
                real td = rmax((real)0.05, bestBarrierDist);
                /* (vr - r*2*dvr/trr + vb - vi) / td, CellProcessor.cuh:272,
                 * with vr + vb - vi = 0 cancelled algebraically */
                F = vdiv(vmul(r, -2 * dvr / trr), td);
            }
        }
        F = vadd(F, vadd(vmul(Fp, (real)p->pressureStrength), vmul(Fv, (real)p->viscosityStrength)));
        w->force[i] = F;
        w->posPrime[i] = vadd(pi, dx);
        w->densNew[i] = dens;
        w->best[i] = best;
    }
}

/* collision force of the pair (cell, other) seen from `cell`,
 * CellProcessor.cuh:322-341 */
static vec2 collisionForce(const OracleWorld* w, int64_t cell, int64_t other, vec2 pd, real d)
{
    const AlienPhysicsParams* p = &w->p;
    vec2 vd = vsub(w->vel[cell], w->vel[other]);
    int approaching = vdot(pd, vd) < 0;
    real bf = w->barrier[cell] ? 2 : 1;
    if (vlen(w->vel[cell]) > (real)0.5 && approaching) {
        real ds = d * d + (real)0.25;
        return vmul(vdiv(vmul(pd, vdot(vd, pd)), -2 * ds), bf);
    }
    return vmul(vmul(vnormalized(pd), ((real)p->cellMaxCollisionDistance - vlen(pd)) * (real)p->cellRepulsionStrength), bf);
}

/* ---- collision pair forces, CellProcessor.cuh:285-365 with
 *      CellMap::executeForEach Map.cuh:175-196 (D1, D2, D5) */
static void collisionPhase(OracleWorld* w)
{
    const AlienPhysicsParams* p = &w->p;
    const real R = (real)p->cellMaxCollisionDistance;
    const int radiusInt = (int)ceilf(p->cellMaxCollisionDistance);
    const real minDist = (real)p->cellMinDistance;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < w->nCells; ++i) {
        if (!w->alive[i]) continue;
        vec2 pi = w->pos[i];
        /* zone values at the cell, CellProcessor.cuh:344-353 */
        const real fusionVelocity = zoneParam(w, ZF_CELL_FUSION_VELOCITY, pi, p->cellFusionVelocity, 0);
        const real maxBindingEnergy = zoneParam(w, ZF_CELL_MAX_BINDING_ENERGY, pi, p->cellMaxBindingEnergy, 0);
        vec2 F = v2(0, 0), dx = v2(0, 0);
        int32_t best = -1;
        uint64_t bestId = UINT64_MAX;
        int cx = floorInt(pi.x), cy = floorInt(pi.y);
        for (int dyy = -radiusInt; dyy <= radiusInt; ++dyy)
            for (int dxx = -radiusInt; dxx <= radiusInt; ++dxx) {
                int sx = wrapInt(cx + dxx, w->W), sy = wrapInt(cy + dyy, w->H);
                int32_t j = w->slotHead[sx + sy * w->W];
                for (int level = 0; level < SLOT_SCAN_LEVELS && j >= 0; ++level, j = w->slotNext[j]) {
                    if (j == i) continue;
                    if (!(vlen(vsub(w->pos[j], pi)) <= R)) continue; /* uncorrected, Map.cuh:189 */
                    vec2 pd = correctDirection(w, vsub(pi, w->pos[j]));
                    real d = vlen(pd);
                    if (!w->barrier[i] && d < minDist) dx = vadd(dx, vmul(pd, minDist / 5));
                    if (isBonded(w, i, j)) continue;
                    /* the pair force is applied to both cells by whichever
                     * cell scans: here as gather, F_i += f(i,j) - f(j,i) */
                    F = vadd(F, collisionForce(w, i, j, pd, d));
                    vec2 vd = vsub(w->vel[i], w->vel[j]);
                    int approaching = vdot(pd, vd) < 0;
                    if (w->numConn[i] < w->maxConn[i] && w->numConn[j] < w->maxConn[j]
                        && vlen(vd) >= fusionVelocity && approaching
                        && w->energy[i] <= maxBindingEnergy && w->energy[j] <= maxBindingEnergy
                        && !w->barrier[i] && !w->barrier[j]) {
                        if (w->id[j] < bestId) {
                            bestId = w->id[j];
                            best = j;
                        }
                    }
                }
            }
        /* contributions made by the scans of other cells that see i */
        if (w->slotRank[i] < SLOT_SCAN_LEVELS) {
            for (int dyy = -radiusInt; dyy <= radiusInt; ++dyy)
                for (int dxx = -radiusInt; dxx <= radiusInt; ++dxx) {
                    int sx = wrapInt(cx + dxx, w->W), sy = wrapInt(cy + dyy, w->H);
                    for (int32_t j = w->slotHead[sx + sy * w->W]; j >= 0; j = w->slotNext[j]) {
                        if (j == i) continue;
                        if (!(vlen(vsub(pi, w->pos[j])) <= R)) continue;
                        if (isBonded(w, j, i)) continue;
                        vec2 pdj = correctDirection(w, vsub(w->pos[j], pi));
                        F = vsub(F, collisionForce(w, j, i, pdj, vlen(pdj)));
                    }
                }
        }
        w->force[i] = F;
        w->posPrime[i] = vadd(pi, dx);
        w->densNew[i] = w->density[i];
        w->best[i] = best;
    }
}

/* ---- bond forces, CellProcessor::calcConnectionForces
 *      CellProcessor.cuh:408-491; positions from `P`, angle terms scattered
 *      into w->angleAcc (D2) */
static void bondForces(OracleWorld* w, const vec2* P, int considerAngles, vec2* out)
{
    const real minDist = (real)w->p.cellMinDistance;
    for (int64_t i = 0; i < w->nCells; ++i) w->angleAcc[i] = v2(0, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < w->nCells; ++i) {
        vec2 F = v2(0, 0);
        int n = w->numConn[i];
        if (w->alive[i] && n > 0 && !w->barrier[i]) {
            vec2 prevDisp = correctDirection(w, vsub(P[w->bond[i][n - 1]], P[i]));
            real s2 = w->stiffness[i] * w->stiffness[i];
            for (int k = 0; k < n; ++k) {
                int32_t j = w->bond[i][k];
                real sj2 = w->stiffness[j] * w->stiffness[j];
                vec2 disp = correctDirection(w, vsub(P[j], P[i]));
                real dist = vlen(disp);
                real dev = dist - w->bondDist[i][k];
                F = vadd(F, vmul(vnormalized(disp), dev * (s2 + sj2) / 6));
                if (considerAngles && (n > 2 || (n == 2 && k == 0))) {
                    int last = (k + n - 1) % n;
                    int32_t jl = w->bond[i][last];
                    int tri = isBonded(w, j, jl);
                    if (!tri) {
                        real a = angleOfVector(disp), pa = angleOfVector(prevDisp);
                        real act = subtractAngle(a, pa);
                        if (act < 0) continue;
                        real ref = w->bondAngle[i][k];
                        real strength = R_ABS(ref - act) / 2000 * s2;
                        vec2 f1 = rotCW(vmul(vdiv(vnormalized(disp), rmax(vlen(disp), minDist)), strength));
                        vec2 f2 = rotCCW(vmul(vdiv(vnormalized(prevDisp), rmax(vlen(prevDisp), minDist)), strength));
                        if (ref < act) {
                            f1 = vmul(f1, -1);
                            f2 = vmul(f2, -1);
                        }
                        if (!w->barrier[j]) {
#pragma omp atomic
                            w->angleAcc[j].x += f1.x;
#pragma omp atomic
                            w->angleAcc[j].y += f1.y;
                        }
                        if (!w->barrier[jl]) {
#pragma omp atomic
                            w->angleAcc[jl].x += f2.x;
#pragma omp atomic
                            w->angleAcc[jl].y += f2.y;
                        }
                        F = vsub(F, vadd(f1, f2));
                    }
                }
                prevDisp = disp;
            }
        }
        out[i] = F;
    }
    for (int64_t i = 0; i < w->nCells; ++i) out[i] = vadd(out[i], w->angleAcc[i]);
}

/* ---- particle movement + collision, RadiationProcessor.cuh:61-170 (D4) */
static void particlePhase(OracleWorld* w, int64_t nOrigParts)
{
    const AlienPhysicsParams* p = &w->p;
    for (int64_t q = 0; q < nOrigParts; ++q) {
        if (!w->palive[q]) continue;
        if (p->numZones > 0) w->pvel[q] = vadd(w->pvel[q], flowAcceleration(w, w->ppos[q])); /* FlowFieldKernels.cu:71-87 */
        w->ppos[q] = correctPosition(w, vadd(w->ppos[q], vmul(w->pvel[q], (real)p->timestepSize)));
    }
    for (int64_t q = 0; q < nOrigParts; ++q) {
        w->ptarget[q] = -1;
        w->pincoming[q] = 0;
        w->mergeE[q] = 0;
        w->mergeMx[q] = 0;
        w->mergeMy[q] = 0;
        if (!w->palive[q]) continue;
        int32_t o = w->pmap[slotOfPos(w, w->ppos[q])];
        if (o >= 0 && o != q && vlen2(vsub(w->ppos[q], w->ppos[o])) < (real)0.5) w->ptarget[q] = o;
    }
    for (int64_t q = 0; q < nOrigParts; ++q) {
        int32_t o = w->ptarget[q];
        if (o < 0 || w->ptarget[o] >= 0) continue;
        if (!(w->penergy[q] > NEAR_ZERO && w->penergy[o] > NEAR_ZERO)) continue;
        w->pincoming[o] = 1;
        w->mergeE[o] += w->penergy[q];
        w->mergeMx[o] += w->penergy[q] * w->pvel[q].x;
        w->mergeMy[o] += w->penergy[q] * w->pvel[q].y;
        w->palive[q] = 0;
    }
    for (int64_t q = 0; q < nOrigParts; ++q) {
        if (!w->palive[q] || !w->pincoming[q]) continue;
        real e = w->penergy[q] + w->mergeE[q];
        w->pvel[q] = v2((w->penergy[q] * w->pvel[q].x + w->mergeMx[q]) / e, (w->penergy[q] * w->pvel[q].y + w->mergeMy[q]) / e);
        w->penergy[q] = e;
        w->plastAbsorbed[q] = UINT64_MAX;
    }
    for (int64_t i = 0; i < w->nCells; ++i) w->energyAdd[i] = 0;
    for (int64_t q = 0; q < nOrigParts; ++q) {
        if (!w->palive[q] || w->ptarget[q] >= 0 || w->pincoming[q]) continue;
        int32_t c = w->slotHead[slotOfPos(w, vadd(w->ppos[q], w->pvel[q]))];
        if (c < 0) continue;
        if (w->barrier[c]) {
            vec2 vr = vsub(w->pvel[q], w->vel[c]);
            vec2 r = correctDirection(w, vsub(w->ppos[q], w->posPrime[c]));
            real dvr = vdot(vr, r);
            if (dvr < 0) {
                real trr = rmax((real)0.1, vlen2(r));
                w->pvel[q] = vadd(vsub(vr, vmul(r, 2 * dvr / trr)), w->vel[c]);
            }
        } else {
            if (w->plastAbsorbed[q] == w->id[c]) continue;
            int cc = w->color[c] % ALIEN_B200_MAX_COLORS;
            real absorption = zoneParam(w, ZF_RADIATION_ABSORPTION, w->posPrime[c], p->radiationAbsorption[cc], cc);
            if (absorption < NEAR_ZERO) continue;
            real transfer = w->penergy[q] * absorption;
            if (w->penergy[q] < (real)0.01f) transfer = w->penergy[q];
            w->energyAdd[c] += transfer;
            w->penergy[q] -= transfer;
            if (w->penergy[q] < NEAR_ZERO)
                w->palive[q] = 0;
            else
                w->plastAbsorbed[q] = w->id[c];
        }
    }
    for (int64_t i = 0; i < w->nCells; ++i) w->energy[i] += w->energyAdd[i];
}

/* ---- RadiationProcessor::splitting, RadiationProcessor.cuh:172-204 */
static void splittingPhase(OracleWorld* w, int64_t nOrigParts, uint64_t T)
{
    const AlienPhysicsParams* p = &w->p;
    for (int64_t q = 0; q < nOrigParts; ++q) {
        if (!w->palive[q]) continue;
        if (draw(w->pid[q], T, SITE_SPLIT) >= 0.01f) continue;
        if (w->penergy[q] > (real)p->particleSplitEnergy[w->pcolor[q] % ALIEN_B200_MAX_COLORS]) {
            w->penergy[q] *= (real)0.5;
            vec2 vp = unitVectorOfAngle((real)draw(w->pid[q], T, SITE_SPLIT_ANGLE) * 360);
            vec2 otherPos = correctPosition(w, vadd(w->ppos[q], vdiv(vp, 5)));
            w->ppos[q] = correctPosition(w, vsub(w->ppos[q], vdiv(vp, 5)));
            vp = vmul(vp, (real)p->radiationVelocityPerturbation / (w->penergy[q] + 1));
            vec2 otherVel = vadd(w->pvel[q], vp);
            w->pvel[q] = vsub(w->pvel[q], vp);
            createParticle(w, otherPos, otherVel, w->pcolor[q], w->penergy[q]);
        }
    }
}

/* ---- CellConnectionProcessor::tryAddConnectionOneWay,
 *      CellConnectionProcessor.cuh:274-427 (angle alignment None), reading
 *      partner bond lists as they stand before the phase (D4) */
typedef struct {
    int n;
    int32_t b[MAX_BONDS];
    real d[MAX_BONDS], a[MAX_BONDS];
} BondList;

/* bond list of cell c as stored (the fusion pass reads the lists before
 * any of its own additions, D4) */
static BondList bondListOf(const OracleWorld* w, int64_t c)
{
    BondList l;
    l.n = w->numConn[c];
    for (int k = 0; k < MAX_BONDS; ++k) {
        l.b[k] = w->bond[c][k];
        l.d[k] = w->bondDist[c][k];
        l.a[k] = w->bondAngle[c][k];
    }
    return l;
}

static int wouldOverlap(const OracleWorld* w, int64_t c1, vec2 otherPos)
{
    /* CellConnectionProcessor.cuh:476-500 */
    int n = w->numConn[c1];
    if (n < 2) return 0;
    for (int k = 0; k < n; ++k) {
        int32_t cc = w->bond[c1][k], nc = w->bond[c1][(k + 1) % n];
        int both = 0;
        for (int m = 0; m < w->numConn[cc]; ++m)
            if (w->bond[cc][m] == nc) {
                both = 1;
                break;
            }
        if (!both) continue;
        if (crossing(w->pos[c1], otherPos, w->pos[cc], w->pos[nc])) return 1;
    }
    return 0;
}

static int tryAddOneWay(const OracleWorld* w, int64_t c1, int64_t c2, vec2 posDelta, BondList* out)
{
    *out = bondListOf(w, c1);
    if (out->n == MAX_BONDS) return 0;
    if (wouldOverlap(w, c1, w->pos[c2])) return 0;
    real newAngle = angleOfVector(posDelta);
    real desired = vlen(posDelta);
    if (out->n == 0) {
        out->n = 1;
        out->b[0] = (int32_t)c2;
        out->d[0] = desired;
        out->a[0] = 360;
        return 1;
    }
    if (out->n == 1) {
        vec2 dc = correctDirection(w, vsub(w->pos[out->b[0]], w->pos[c1]));
        real prevAngle = angleOfVector(dc);
        real diff = newAngle - prevAngle;
        if (diff < 0) diff += (real)360.0;
        if (R_ABS(diff) < NEAR_ZERO || R_ABS(diff - 360) < NEAR_ZERO || R_ABS(diff + 360) < NEAR_ZERO) return 0;
        out->a[1] = diff;
        out->a[0] = 360 - diff;
        out->n = 2;
        out->b[1] = (int32_t)c2;
        out->d[1] = desired;
        return 1;
    }
    int n = out->n, index = 0;
    real prevAngle = 0, nextAngle = 0;
    for (; index < n; ++index) {
        int prevIndex = (index + n - 1) % n;
        prevAngle = angleOfVector(correctDirection(w, vsub(w->pos[out->b[prevIndex]], w->pos[c1])));
        nextAngle = angleOfVector(correctDirection(w, vsub(w->pos[out->b[index]], w->pos[c1])));
        if (isAngleInBetween(prevAngle, nextAngle, newAngle) || prevIndex == index) break;
    }
    if (index == n) return 0; /* no gap found: the reference would read past the list */
    real refAngle = out->a[index];
    real d1 = subtractAngle(newAngle, prevAngle), d2 = subtractAngle(nextAngle, prevAngle);
    real fraction = d2 != 0 ? d1 / d2 : (real)0.5;
    real afp = rmin(refAngle * fraction, refAngle);
    if (afp < NEAR_ZERO) return 0;
    if (index == 0) index = n;
    for (int j = n; j > index; --j) {
        out->b[j] = out->b[j - 1];
        out->d[j] = out->d[j - 1];
        out->a[j] = out->a[j - 1];
    }
    out->b[index] = (int32_t)c2;
    out->d[index] = desired;
    out->a[index] = afp;
    out->a[(index + 1) % (n + 1)] = refAngle - afp;
    out->n = n + 1;
    return 1;
}

/* ---- CellConnectionProcessor::deleteConnectionOneWay,
 *      CellConnectionProcessor.cuh:429-448 */
static void deleteOneWay(OracleWorld* w, int64_t c, int32_t other)
{
    int n = w->numConn[c];
    for (int k = 0; k < n; ++k) {
        if (w->bond[c][k] != other) continue;
        real add = w->bondAngle[c][k];
        for (int j = k; j < n - 1; ++j) {
            w->bond[c][j] = w->bond[c][j + 1];
            w->bondDist[c][j] = w->bondDist[c][j + 1];
            w->bondAngle[c][j] = w->bondAngle[c][j + 1];
        }
        if (k < n - 1)
            w->bondAngle[c][k] += add;
        else
            w->bondAngle[c][0] += add;
        w->bond[c][n - 1] = -1;
        w->numConn[c] = (uint8_t)(n - 1);
        return;
    }
}

/* ---- stable compaction of cells and particles (D6), replacing
 *      cudaCleanupPointerArray / cudaCleanupCellsStep1/2,
 *      GarbageCollectorKernels.cuh:12-48, GarbageCollectorKernels.cu:16-52 */
static void compact(OracleWorld* w)
{
    int32_t* remap = malloc(sizeof(int32_t) * (size_t)(w->nCells > 0 ? w->nCells : 1));
    int64_t n = 0;
    for (int64_t i = 0; i < w->nCells; ++i) remap[i] = w->alive[i] ? (int32_t)n++ : -1;
    if (n != w->nCells) {
        for (int64_t i = 0; i < w->nCells; ++i) {
            if (!w->alive[i]) continue;
            int64_t t = remap[i];
            w->id[t] = w->id[i]; w->pos[t] = w->pos[i]; w->vel[t] = w->vel[i]; w->energy[t] = w->energy[i];
            w->stiffness[t] = w->stiffness[i]; w->density[t] = w->density[i]; w->color[t] = w->color[i];
            w->maxConn[t] = w->maxConn[i]; w->numConn[t] = w->numConn[i]; w->barrier[t] = w->barrier[i];
            w->alive[t] = 1; w->livingState[t] = w->livingState[i]; w->age[t] = w->age[i];
            w->activationTime[t] = w->activationTime[i]; w->creatureId[t] = w->creatureId[i];
            w->cellFunction[t] = w->cellFunction[i]; w->cold[t] = w->cold[i]; w->forceOld[t] = w->forceOld[i];
            for (int k = 0; k < MAX_BONDS; ++k) {
                w->bond[t][k] = w->bond[i][k];
                w->bondDist[t][k] = w->bondDist[i][k];
                w->bondAngle[t][k] = w->bondAngle[i][k];
            }
        }
        for (int64_t t = 0; t < n; ++t)
            for (int k = 0; k < w->numConn[t]; ++k) w->bond[t][k] = remap[w->bond[t][k]];
        w->nCells = n;
    }
    free(remap);
    int64_t m = 0;
    for (int64_t q = 0; q < w->nParts; ++q) {
        if (!w->palive[q]) continue;
        if (m != q) {
            w->pid[m] = w->pid[q]; w->ppos[m] = w->ppos[q]; w->pvel[m] = w->pvel[q];
            w->penergy[m] = w->penergy[q]; w->pcolor[m] = w->pcolor[q]; w->pselected[m] = w->pselected[q];
            w->plastAbsorbed[m] = w->plastAbsorbed[q];
        }
        w->palive[m] = 1;
        ++m;
    }
    w->nParts = m;
}

/* ---- one timestep ---- */
/* The neuron cell function: CellFunctionProcessor::collectCellFunctionOperations
 * (CellFunctionProcessor.cuh:33-50) picks cells whose execution order number
 * is timestep % cellNumExecutionOrderNumbers, not under construction or
 * activating, activation time 0; NeuronProcessor::processCell
 * (NeuronProcessor.cuh:33-74) with calcInputSignal (CellFunctionProcessor.cuh
 * :128-164: bonded inputs of the input execution order number, each channel
 * clamped to [-10, 10] after every addition, in bond order) and
 * updateInvocationState (:176-186); activations NeuronProcessor.cuh:76-90.
 * Weights and biases are read from the auxiliary data at
 * NeuronTO.weightsAndBiasesDataIndex (TOs.cuh:45-49).  Inputs of a running
 * neuron never run in the same step, so signals are read and written in one
 * pass. */
static real neuronActivation(int function, real x)
{
    switch (function) {
    case 0: return 2 / (1 + exp(-x)) - 1;
    case 1: return x >= (real)NEAR_ZERO ? 1 : 0;
    case 2: return x < -1 ? -1 : (x > 1 ? 1 : x);
    case 3: return fabs(x) < 1 ? fabs(x) : 1;
    case 4: return exp(-2 * x * x);
    }
    return 0;
}

static void neuronPhase(OracleWorld* w, uint64_t T)
{
    const int64_t N = w->nCells;
    const uint64_t orders = (uint64_t)(w->p.cellNumExecutionOrderNumbers > 0 ? w->p.cellNumExecutionOrderNumbers : 1);
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i] || w->cellFunction[i] != 0) continue;
        AlienCellTO* me = &w->cold[i];
        if ((uint64_t)me->executionOrderNumber != T % orders) continue;
        int ls = w->livingState[i];
        if (ls == ALIEN_B200_LIVING_UNDER_CONSTRUCTION || ls == ALIEN_B200_LIVING_ACTIVATING || w->activationTime[i] != 0) continue;
        real in[ALIEN_B200_MAX_CHANNELS] = {0};
        uint8_t origin = 0;
        real tx = 0, ty = 0;
        int inputOrder = me->inputExecutionOrderNumber;
        if (inputOrder != -1 && inputOrder != (int)me->executionOrderNumber) {
            int sensors = 0;
            for (int k = 0; k < w->numConn[i]; ++k) {
                int32_t j = w->bond[i][k];
                const AlienCellTO* o = &w->cold[j];
                int lsj = w->livingState[j];
                if (o->outputBlocked || lsj == ALIEN_B200_LIVING_UNDER_CONSTRUCTION || lsj == ALIEN_B200_LIVING_ACTIVATING) continue;
                if ((int)o->executionOrderNumber != inputOrder) continue;
                for (int c = 0; c < ALIEN_B200_MAX_CHANNELS; ++c) {
                    real v = in[c] + (real)o->signal.channels[c];
                    in[c] = v < -10 ? -10 : (v > 10 ? 10 : v);
                }
                if (o->signal.origin == 1) {
                    origin = 1;
                    tx += o->signal.targetX;
                    ty += o->signal.targetY;
                    ++sensors;
                }
            }
            if (sensors > 0) {
                tx /= sensors;
                ty /= sensors;
            }
        }
        if (me->cellFunctionUsed == 0)
            for (int c = 0; c < ALIEN_B200_MAX_CHANNELS - 1; ++c)
                if (in[c] != 0) {
                    me->cellFunctionUsed = 1;
                    break;
                }
        float wb[ALIEN_B200_MAX_CHANNELS * (ALIEN_B200_MAX_CHANNELS + 1)];
        if (me->cellFunctionData[0] > w->nAux || w->nAux - me->cellFunctionData[0] < sizeof(wb)) continue;
        memcpy(wb, w->aux + me->cellFunctionData[0], sizeof(wb));
        int32_t act[ALIEN_B200_MAX_CHANNELS];
        memcpy(act, (const uint8_t*)me->cellFunctionData + 8, sizeof(act));
        real out[ALIEN_B200_MAX_CHANNELS];
        for (int r = 0; r < ALIEN_B200_MAX_CHANNELS; ++r) {
            real sum = wb[ALIEN_B200_MAX_CHANNELS * ALIEN_B200_MAX_CHANNELS + r];
            for (int c = 0; c < ALIEN_B200_MAX_CHANNELS; ++c) sum += (real)wb[r * ALIEN_B200_MAX_CHANNELS + c] * in[c];
            out[r] = neuronActivation(act[r], sum);
        }
        for (int r = 0; r < ALIEN_B200_MAX_CHANNELS; ++r) me->signal.channels[r] = (float)out[r];
        me->signal.origin = origin;
        me->signal.targetX = (float)tx;
        me->signal.targetY = (float)ty;
        ++w->neuronActivity[w->color[i] % ALIEN_B200_MAX_COLORS]; /* NeuronProcessor.cuh:70 */
    }
}

/* CellFunctionProcessor::resetFetchedSignals (CellFunctionProcessor.cuh:69-112),
 * called by the friction kernel after the cell functions (SimulationKernels.cu
 * :153-158): cells without function lose their signal channels every step;
 * cells with a function in the step after the last of their readers ran. */
static void signalReset(OracleWorld* w, uint64_t T)
{
    const int64_t N = w->nCells;
    const int orders = w->p.cellNumExecutionOrderNumbers > 0 ? w->p.cellNumExecutionOrderNumbers : 1;
    const int current = (int)(T % (uint64_t)orders);
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i]) continue;
        AlienCellTO* me = &w->cold[i];
        int reset = me->cellFunction == 11; /* CellFunction_None */
        if (!reset) {
            int own = me->executionOrderNumber, maxOther = -1;
            if (!me->outputBlocked) {
                for (int k = 0; k < w->numConn[i]; ++k) {
                    const AlienCellTO* o = &w->cold[w->bond[i][k]];
                    int other = o->executionOrderNumber;
                    if (o->inputExecutionOrderNumber != own) continue;
                    if (maxOther == -1)
                        maxOther = other;
                    else if ((maxOther > own && (other > maxOther || other < own)) || (maxOther < own && other > maxOther && other < own))
                        maxOther = other;
                }
            }
            reset = (maxOther == -1 && current == (own + 1) % orders) || (maxOther != -1 && maxOther == current);
        }
        if (reset)
            for (int c = 0; c < ALIEN_B200_MAX_CHANNELS; ++c) me->signal.channels[c] = 0;
    }
}

/* ---- rigidity clusters (ClusterProcessor.cuh:8-168, every third step after
 *      friction, SimulationKernelsLauncher.cu:74-83).  Clusters by the same
 *      synchronous Shiloach-Vishkin rounds as the engine (gather: shortcut
 *      and aggressive hooking from the previous labels; scatter: hooking of
 *      the cell's label by minima; at most CLUSTER_ROUNDS rounds, ended by a
 *      round that changes nothing), offsets from the label cell by minimal
 *      image, sums in double (the reference: three lock-free label walks,
 *      float atomics, and a world-thirds seam correction that agrees with
 *      the minimal image for clusters smaller than a third of the world) */
#define CLUSTER_ROUNDS 12
static int rigidityEnabled(const AlienPhysicsParams* p) /* SimulationKernelsLauncher.cu:99-107 */
{
    for (int i = 0; i < p->numZones; ++i)
        if (p->zones[i].rigidity != 0.0f) return 1;
    return p->rigidity != 0.0f;
}

static void rigidityPhase(OracleWorld* w)
{
    const AlienPhysicsParams* p = &w->p;
    const int64_t N = w->nCells;
    if (N == 0) return;
    int32_t* lab[2] = {malloc(sizeof(int32_t) * (size_t)N), malloc(sizeof(int32_t) * (size_t)N)};
    for (int64_t i = 0; i < N; ++i) lab[0][i] = (int32_t)i;
    int cur = 0;
    for (int r = 0; r < CLUSTER_ROUNDS; ++r) {
        const int32_t* f = lab[r & 1];
        int32_t* g = lab[(r + 1) & 1];
        int changed = 0;
        for (int64_t i = 0; i < N; ++i) {
            if (!w->alive[i]) continue;
            int32_t m = f[f[i]] < f[i] ? f[f[i]] : f[i];
            for (int k = 0; k < w->numConn[i]; ++k) {
                int32_t x = f[f[w->bond[i][k]]];
                if (x < m) m = x;
            }
            g[i] = m;
            changed |= m != f[i];
        }
        for (int64_t i = 0; i < N; ++i) {
            if (!w->alive[i]) continue;
            int32_t m = f[i];
            for (int k = 0; k < w->numConn[i]; ++k) {
                int32_t x = f[f[w->bond[i][k]]];
                if (x < m) m = x;
            }
            if (m < g[f[i]]) {
                g[f[i]] = m;
                changed = 1;
            }
        }
        cur = (r + 1) & 1;
        if (!changed) break;
    }
    const int32_t* cl = lab[cur];
    vec2* velSum = calloc((size_t)N, sizeof(vec2));
    vec2* relSum = calloc((size_t)N, sizeof(vec2));
    real* mass = calloc((size_t)N, sizeof(real));
    real* mom = calloc((size_t)N, sizeof(real));
    int64_t* count = calloc((size_t)N, sizeof(int64_t));
    vec2* rel = malloc(sizeof(vec2) * (size_t)N);
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i]) continue;
        rel[i] = correctDirection(w, vsub(w->pos[i], w->pos[cl[i]]));
        velSum[cl[i]] = vadd(velSum[cl[i]], w->vel[i]);
        relSum[cl[i]] = vadd(relSum[cl[i]], rel[i]);
        count[cl[i]] += 1;
    }
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i]) continue;
        const int32_t c = cl[i];
        vec2 cv = vdiv(velSum[c], (real)count[c]), r = vsub(rel[i], vdiv(relSum[c], (real)count[c]));
        vec2 dv = vsub(w->vel[i], cv);
        mass[c] += r.x * r.x + r.y * r.y;     /* Math::lengthSquared */
        mom[c] += r.x * dv.y - r.y * dv.x;     /* Physics::angularMomentum */
    }
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i]) continue;
        const int32_t c = cl[i];
        vec2 cv = vdiv(velSum[c], (real)count[c]), r = vsub(rel[i], vdiv(relSum[c], (real)count[c]));
        real av = R_ABS(mass[c]) < NEAR_ZERO ? 0 : mom[c] / mass[c] * RAD_TO_DEG; /* Physics.cuh:191-197 */
        real rigidity = zoneParam(w, ZF_RIGIDITY, w->pos[i], p->rigidity, 0) * w->stiffness[i] * w->stiffness[i];
        vec2 tangential = v2(cv.x - av * r.y * DEG_TO_RAD, cv.y + av * r.x * DEG_TO_RAD); /* Physics.cuh:181-184 */
        w->vel[i] = vadd(vmul(w->vel[i], 1 - rigidity), vmul(tangential, rigidity));
    }
    free(lab[0]); free(lab[1]); free(velSum); free(relSum); free(mass); free(mom); free(count); free(rel);
}

static void stepOnce(OracleWorld* w)
{
    const AlienPhysicsParams* p = &w->p;
    const uint64_t T = w->timestep;
    const int considerAngles = (T % 3 == 0);        /* SimulationKernelsLauncher.cu:31 */
    const int considerInnerFriction = (T % 3 == 0); /* :32 */
    const real dt = (real)p->timestepSize;
    const int64_t nOrigParts = w->nParts; /* SimulationData::prepareForNextTimestep :46 */
    const int64_t N = w->nCells;

    /* RadiationProcessor::calcActiveSources (physics_init, SimulationKernels.cu:23-27) */
    w->activeSources = calcActiveSources(w);
    w->backflowSum = 0;

    /* cudaNextTimestep_physics_init + fillMaps: SimulationKernels.cu:23-34 */
    for (int64_t i = 0; i < N; ++i) {
        w->force[i] = v2(0, 0);
        w->delAll[i] = w->delCell[i] = w->detachFlag[i] = w->setDying[i] = w->newlyDying[i] = 0;
        w->newPartner[i] = -1;
    }
    buildCellMap(w);
    radiationPhase(w, T);

    /* physics_calcFluidForces / calcCollisionForces: SimulationKernels.cu:36-50 */
    if (p->motionType == ALIEN_B200_MOTION_FLUID)
        fluidPhase(w);
    else
        collisionPhase(w);
    /* RadiationProcessor::updateMap (last writer = highest index, D5) */
    for (int64_t q = 0; q < nOrigParts; ++q) {
        w->pslot[q] = -1;
        if (!w->palive[q]) continue;
        w->pslot[q] = slotOfPos(w, w->ppos[q]);
        w->pmap[w->pslot[q]] = (int32_t)q;
    }

    /* physics_applyForces: checkForces + applyForces (CellProcessor.cuh:367-406) */
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i]) continue;
        if (p->motionType == ALIEN_B200_MOTION_FLUID) w->density[i] = w->densNew[i];
        if (w->barrier[i]) continue;
        int c = w->color[i] % ALIEN_B200_MAX_COLORS;
        /* flow fields (cudaApplyFlowFieldSettings, FlowFieldKernels.cu:48-70)
         * add to the pair force at the cell after the overlap push */
        vec2 F = w->force[i];
        real maxForce = p->cellMaxForce[c];
        if (p->numZones > 0) {
            F = vadd(F, flowAcceleration(w, w->posPrime[i]));
            maxForce = zoneParam(w, ZF_CELL_MAX_FORCE, w->posPrime[i], maxForce, c);
        }
        if (vlen(F) > maxForce) {
            if (draw(w->id[i], T, SITE_FORCE_DECAY) < p->cellMaxForceDecayProb) w->delAll[i] = 1;
        }
        vec2 v = vadd(w->vel[i], F);
        if (vlen(v) > (real)p->cellMaxVelocity) v = vmul(vnormalized(v), (real)p->cellMaxVelocity);
        w->vel[i] = v;
    }
    particlePhase(w, nOrigParts);
    for (int64_t q = 0; q < nOrigParts; ++q)
        if (w->pslot[q] >= 0) w->pmap[w->pslot[q]] = -1;

    /* calcConnectionForces #1 at the overlap-corrected positions */
    vec2* F1 = w->forceOld;
    bondForces(w, w->posPrime, considerAngles, F1);
    /* verletPositionUpdate + checkConnections (CellProcessor.cuh:493-544) */
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i]) continue;
        vec2 np;
        if (w->barrier[i])
            np = vadd(w->posPrime[i], vmul(w->vel[i], dt));
        else
            np = vadd(vadd(w->posPrime[i], vmul(w->vel[i], dt)), vmul(F1[i], dt * dt / 2));
        w->pos[i] = correctPosition(w, np);
    }
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i] || w->barrier[i]) continue;
        int destroy = 0;
        for (int k = 0; k < w->numConn[i]; ++k) {
            vec2 disp = correctDirection(w, vsub(w->pos[w->bond[i][k]], w->pos[i]));
            if (vlen(disp) > (real)p->cellMaxBindingDistance[w->color[i] % ALIEN_B200_MAX_COLORS]) destroy = 1;
        }
        if (destroy) {
            w->delAll[i] = 1;
            for (int k = 0; k < w->numConn[i]; ++k) w->detachFlag[w->bond[i][k]] = 1;
        }
    }
    for (int64_t i = 0; i < N; ++i)
        if (w->alive[i] && w->detachFlag[i]) w->livingState[i] = ALIEN_B200_LIVING_DETACHING;
    splittingPhase(w, nOrigParts, T);

    /* calcConnectionForces #2 + verletVelocityUpdate (CellProcessor.cuh:546-559) */
    vec2* F2 = w->force;
    bondForces(w, w->pos, considerAngles, F2);
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i] || w->barrier[i]) continue;
        w->vel[i] = vadd(w->vel[i], vmul(vdiv(vadd(F2[i], F1[i]), 2), dt));
    }

    /* cellFunction_prepare_substep1/2: aging + living-state transition
     * (CellProcessor.cuh:561-676); cell functions themselves are not part of
     * the physics stage */
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i] || w->barrier[i]) continue;
        ++w->age[i];
        if (w->livingState[i] == ALIEN_B200_LIVING_READY && w->activationTime[i] > 0) --w->activationTime[i];
    }
    int32_t* nextState = malloc(sizeof(int32_t) * (size_t)(N > 0 ? N : 1));
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i]) continue;
        int sameDetaching = 0, otherDetaching = 0, sameReviving = 0, activating = 0;
        for (int k = 0; k < w->numConn[i]; ++k) {
            int32_t j = w->bond[i][k];
            int ls = w->livingState[j];
            if (w->creatureId[j] == w->creatureId[i]) {
                if (ls == ALIEN_B200_LIVING_DETACHING) sameDetaching = 1;
                else if (ls == ALIEN_B200_LIVING_REVIVING) sameReviving = 1;
                else if (ls == ALIEN_B200_LIVING_ACTIVATING) activating = 1;
            } else if (ls == ALIEN_B200_LIVING_DETACHING)
                otherDetaching = 1;
        }
        int orig = w->livingState[i], ls = orig;
        int dc = p->cellDeathConsequences;
        if (w->barrier[i])
            ls = ALIEN_B200_LIVING_READY;
        else if (orig == ALIEN_B200_LIVING_ACTIVATING)
            ls = ALIEN_B200_LIVING_READY;
        else if (orig == ALIEN_B200_LIVING_REVIVING)
            ls = ALIEN_B200_LIVING_READY;
        else if (orig == ALIEN_B200_LIVING_UNDER_CONSTRUCTION) {
            if (activating) ls = ALIEN_B200_LIVING_ACTIVATING;
            if (otherDetaching && dc != ALIEN_B200_DEATH_NONE) ls = ALIEN_B200_LIVING_DETACHING;
        } else if (orig == ALIEN_B200_LIVING_DETACHING) {
            if (sameReviving && dc == ALIEN_B200_DEATH_DETACHED_PARTS_DIE) ls = ALIEN_B200_LIVING_REVIVING;
            if (dc == ALIEN_B200_DEATH_NONE) ls = ALIEN_B200_LIVING_READY;
        } else if (orig == ALIEN_B200_LIVING_READY) {
            /* the self-replicating-constructor exception (GenomeDecoder) needs
             * cell functions, which are outside the physics stage */
            if (sameDetaching && dc != ALIEN_B200_DEATH_NONE) ls = ALIEN_B200_LIVING_DETACHING;
        }
        nextState[i] = ls;
    }
    for (int64_t i = 0; i < N; ++i)
        if (w->alive[i]) w->livingState[i] = nextState[i];
    free(nextState);

    /* cellFunction_neuron (SimulationKernelsLauncher.cu:56) */
    neuronPhase(w, T);
    signalReset(w, T);

    /* applyInnerFriction (every third step, D4), applyFriction, decay
     * (CellProcessor.cuh:678-858) */
    if (considerInnerFriction) {
        vec2* vnew = malloc(sizeof(vec2) * (size_t)(N > 0 ? N : 1));
        const real f = (real)p->innerFriction;
        for (int64_t i = 0; i < N; ++i) {
            vnew[i] = w->vel[i];
            if (!w->alive[i] || w->barrier[i]) continue;
            vec2 acc = v2(0, 0);
            for (int k = 0; k < w->numConn[i]; ++k) {
                int32_t j = w->bond[i][k];
                if (w->barrier[j]) continue;
                acc = vadd(acc, vsub(w->vel[j], w->vel[i]));
            }
            vnew[i] = vadd(w->vel[i], vmul(acc, f / 2));
        }
        memcpy(w->vel, vnew, sizeof(vec2) * (size_t)N);
        free(vnew);
    }
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i] || w->barrier[i]) continue;
        w->vel[i] = vmul(w->vel[i], 1 - zoneParam(w, ZF_FRICTION, w->pos[i], p->friction, 0));
    }
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i] || w->barrier[i]) continue;
        int c = w->color[i] % ALIEN_B200_MAX_COLORS;
        if (w->energy[i] > zoneParam(w, ZF_CELL_MAX_BINDING_ENERGY, w->pos[i], p->cellMaxBindingEnergy, 0)) w->delAll[i] = 1;
        int ls = w->livingState[i];
        if (ls == ALIEN_B200_LIVING_DYING || ls == ALIEN_B200_LIVING_DETACHING) {
            if (draw(w->id[i], T, SITE_DEATH) < zoneParam(w, ZF_CELL_DEATH_PROBABILITY, w->pos[i], p->cellDeathProbability[c], c))
                w->delCell[i] = 1;
        }
        int destroy = w->energy[i] < zoneParam(w, ZF_CELL_MIN_ENERGY, w->pos[i], p->cellMinEnergy[c], c);
        int64_t maxAge = p->cellMaxAge[c];
        if (maxAge > 0 && (int64_t)w->age[i] > maxAge) destroy = 1;
        if (destroy) {
            w->setDying[i] = 1;
            w->newlyDying[i] = ls != ALIEN_B200_LIVING_DYING;
        }
    }
    for (int64_t i = 0; i < N; ++i)
        if (w->alive[i] && w->setDying[i]) w->livingState[i] = ALIEN_B200_LIVING_DYING;
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i] || !w->newlyDying[i]) continue;
        for (int k = 0; k < w->numConn[i]; ++k) {
            int32_t j = w->bond[i][k];
            if (w->livingState[j] != ALIEN_B200_LIVING_DYING) w->livingState[j] = ALIEN_B200_LIVING_DETACHING;
        }
    }
    if (T % 3 == 0 && rigidityEnabled(p)) rigidityPhase(w); /* SimulationKernelsLauncher.cu:33, 74-83 */

    /* structuralOperations_substep2..4 (SimulationKernels.cu:167-180): every
     * new bond list is computed from the lists as they stand before the
     * phase, then all are applied (mutual choices pair each cell at most once) */
    typedef struct {
        int64_t c[2];
        BondList l[2];
    } Fusion;
    int64_t nFusions = 0, capFusions = 0;
    Fusion* fusions = NULL;
    for (int64_t i = 0; i < N; ++i) {
        int32_t j = w->best[i];
        if (!w->alive[i] || j < 0 || j <= i || w->best[j] != i) continue;
        int64_t c1 = w->id[i] < w->id[j] ? i : j, c2 = c1 == i ? j : i;
        vec2 pd = correctDirection(w, vsub(w->pos[c2], w->pos[c1]));
        Fusion f;
        f.c[0] = c1;
        f.c[1] = c2;
        if (!tryAddOneWay(w, c1, c2, pd, &f.l[0])) continue;
        if (!tryAddOneWay(w, c2, c1, vmul(pd, -1), &f.l[1])) continue;
        if (nFusions == capFusions) {
            capFusions = capFusions ? 2 * capFusions : 1024;
            fusions = realloc(fusions, sizeof(Fusion) * (size_t)capFusions);
        }
        fusions[nFusions++] = f;
    }
    for (int64_t f = 0; f < nFusions; ++f) {
        for (int s = 0; s < 2; ++s) {
            const int64_t c = fusions[f].c[s];
            const BondList* l = &fusions[f].l[s];
            w->numConn[c] = (uint8_t)l->n;
            for (int k = 0; k < MAX_BONDS; ++k) {
                w->bond[c][k] = k < l->n ? l->b[k] : -1;
                w->bondDist[c][k] = l->d[k];
                w->bondAngle[c][k] = l->a[k];
            }
        }
        w->newPartner[fusions[f].c[0]] = (int32_t)fusions[f].c[1];
        w->newPartner[fusions[f].c[1]] = (int32_t)fusions[f].c[0];
    }
    free(fusions);
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i] || !w->delCell[i]) continue;
        createEnergyParticle(w, w->pos[i], w->vel[i], w->color[i], w->energy[i], w->id[i], SITE_SOURCE_DELETED_CELL);
        w->alive[i] = 0;
    }
    for (int64_t i = 0; i < N; ++i) {
        if (!w->alive[i]) continue;
        int32_t drop[MAX_BONDS];
        int nd = 0;
        for (int k = 0; k < w->numConn[i]; ++k) {
            int32_t j = w->bond[i][k];
            if (!w->alive[j] || ((w->delAll[i] || w->delAll[j]) && j != w->newPartner[i])) drop[nd++] = j;
        }
        for (int k = 0; k < nd; ++k) deleteOneWay(w, i, drop[k]);
    }

    clearCellMap(w);
    compact(w);
    ++w->timestep;
    /* the pool takes the step's backflow; zones and radiation sources move
     * (SimulationParametersUpdateService.cu:52-78) */
    w->externalEnergy += w->backflowSum;
    for (int i = 0; i < p->numRadiationSources; ++i) {
        AlienRadiationSource* r = &w->p.radiationSources[i];
        moveOnTorus(w, &r->posX, &r->posY, r->velX, r->velY, p->timestepSize);
    }
    for (int i = 0; i < p->numZones; ++i) {
        AlienZone* z = &w->p.zones[i];
        moveOnTorus(w, &z->posX, &z->posY, z->velX, z->velY, p->timestepSize);
    }
}

/* the parameters as the steps left them (zone and source positions, the pool) */
void oracle_get_parameters(OracleWorld* w, AlienPhysicsParams* out)
{
    *out = w->p;
    out->externalEnergy = (float)w->externalEnergy;
}

int oracle_step(OracleWorld* w, uint64_t n)
{
    for (uint64_t s = 0; s < n; ++s) stepOnce(w);
    return 0;
}

/* slot (x + y*W) of every live cell in storage order, for map parity */
int64_t oracle_cell_slots(OracleWorld* w, int32_t* out, int64_t cap)
{
    int64_t n = 0;
    for (int64_t i = 0; i < w->nCells; ++i)
        if (w->alive[i]) {
            if (n < cap) out[n] = slotOfPos(w, w->pos[i]);
            ++n;
        }
    return n;
}

/* accumulated neuron activities per color since creation */
void oracle_neuron_activities(OracleWorld* w, uint64_t* out)
{
    for (int c = 0; c < ALIEN_B200_MAX_COLORS; ++c) out[c] = w->neuronActivity[c];
}

void oracle_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
