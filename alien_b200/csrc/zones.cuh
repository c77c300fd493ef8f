// zones.cuh - zones (position-dependent parameters and flow fields),
// radiation sources and the external-energy backflow of new energy
// particles.
//
// SpotCalculator (source/EngineGpuKernels/SpotCalculator.cuh:12-251) blends a
// parameter from its base value into the values of the zones that activate
// it, by each zone's weight at the position: 0 inside the zone's core, rising
// linearly to 1 over the fade-out radius (+1) outside it.  With weights w_i
// in zone order,
//     result = base * prod(w_i) + sum_i v_i (1 - w_i) / (sum_i (1 - w_i) + prod(w_i))
// (the base term is not divided by the sum, as in the reference's mix()).
// Flow fields (FlowFieldKernels.cu:10-89) blend the accelerations of the
// zones with a flow type the same way, from a base of zero.
// createEnergyParticle (RadiationProcessor.cuh:248-364) places a new energy
// particle at an active radiation source chosen in proportion to the
// sources' strengths, with the reference's shapes and velocity rules; its
// random numbers are counter-based draws here (site ranges below).
#pragma once

#include "device_common.cuh"

namespace ab {

enum ZoneField : int {
    kZFriction,
    kZRigidity,
    kZRadiationAbsorption,
    kZRadiationCellAgeStrength,
    kZCellMaxForce,
    kZCellMinEnergy,
    kZCellDeathProbability,
    kZCellFusionVelocity,
    kZCellMaxBindingEnergy,
    kZRadiationDisableSources,
};

template <int F>
__device__ __forceinline__ bool zoneActivated(const AlienZone& z)
{
    switch (F) {
    case kZFriction: return z.frictionActivated;
    case kZRigidity: return z.rigidityActivated;
    case kZRadiationAbsorption: return z.radiationAbsorptionActivated;
    case kZRadiationCellAgeStrength: return z.radiationCellAgeStrengthActivated;
    case kZCellMaxForce: return z.cellMaxForceActivated;
    case kZCellMinEnergy: return z.cellMinEnergyActivated;
    case kZCellDeathProbability: return z.cellDeathProbabilityActivated;
    case kZCellFusionVelocity: return z.cellFusionVelocityActivated;
    case kZCellMaxBindingEnergy: return z.cellMaxBindingEnergyActivated;
    default: return z.radiationDisableSourcesActivated;
    }
}

template <int F>
__device__ __forceinline__ float zoneValue(const AlienZone& z, int color)
{
    switch (F) {
    case kZFriction: return z.friction;
    case kZRigidity: return z.rigidity;
    case kZRadiationAbsorption: return z.radiationAbsorption[color];
    case kZRadiationCellAgeStrength: return z.radiationCellAgeStrength[color];
    case kZCellMaxForce: return z.cellMaxForce[color];
    case kZCellMinEnergy: return z.cellMinEnergy[color];
    case kZCellDeathProbability: return z.cellDeathProbability[color];
    case kZCellFusionVelocity: return z.cellFusionVelocity;
    case kZCellMaxBindingEnergy: return z.cellMaxBindingEnergy;
    default: return z.radiationDisableSources ? 1.0f : 0.0f;
    }
}

// SpotCalculator::calcWeight, SpotCalculator.cuh:183-210; delta = zone - position
__device__ __forceinline__ float zoneWeight(const AlienZone& z, float2 delta)
{
    if (z.shapeType == ALIEN_B200_SHAPE_RECTANGULAR) {
        if (fabsf(delta.x) > z.width / 2 || fabsf(delta.y) > z.height / 2) {
            const float2 d = f2(fmaxf(0.0f, fabsf(delta.x) - z.width / 2), fmaxf(0.0f, fabsf(delta.y) - z.height / 2));
            return fminf(1.0f, len2(d) / (z.fadeoutRadius + 1.0f));
        }
        return 0.0f;
    }
    const float distance = len2(delta);
    return distance < z.coreRadius ? 0.0f : fminf(1.0f, (distance - z.coreRadius) / (z.fadeoutRadius + 1.0f));
}

__device__ __forceinline__ float2 zoneDelta(const AlienZone& z, float2 pos, int W, int H)
{
    return seamDiff2(f2(z.posX, z.posY), pos, W, H);
}

// SpotCalculator::calcParameter (:78-160): the parameter F at the position,
// `base` its base value (of the cell's color where it has one)
template <int F>
__device__ __forceinline__ float zoneParam(const AlienPhysicsParams& p, int W, int H, float2 pos, float base, int color = 0)
{
    if (p.numZones <= 0) return base;
    float baseFactor = 1.0f, sum = 0.0f;
    for (int i = 0; i < p.numZones; ++i) {
        const AlienZone& z = p.zones[i];
        if (!zoneActivated<F>(z)) continue;
        const float w = zoneWeight(z, zoneDelta(z, pos, W, H));
        baseFactor *= w;
        sum += 1.0f - w;
    }
    sum += baseFactor;
    float result = base * baseFactor;
    for (int i = 0; i < p.numZones; ++i) {
        const AlienZone& z = p.zones[i];
        if (!zoneActivated<F>(z)) continue;
        const float w = zoneWeight(z, zoneDelta(z, pos, W, H));
        result += zoneValue<F>(z, color) * (1.0f - w) / sum;
    }
    return result;
}

// Math::rotateClockwise (Math.cuh:171-193, 293-298), angle in degrees
__device__ __forceinline__ float2 rotateClockwiseDeg(float2 v, float angle)
{
    const float a = angle * (kPi / 180.0f);
    const float sn = sinf(a), cs = cosf(a);
    return f2(v.x * cs - v.y * sn, v.x * sn + v.y * cs);
}

// calcAcceleration, FlowFieldKernels.cu:10-44
__device__ __forceinline__ float zoneFlowHeight(const AlienZone& z, float2 pos, int W, int H)
{
    const float h = sqrtf(len2(seamDiff2(pos, f2(z.posX, z.posY), W, H))) * z.flowStrength;
    return z.flowOrientation == 0 ? h : -h;  // Orientation_Clockwise
}
__device__ __forceinline__ float2 zoneFlowAcceleration(const AlienZone& z, float2 pos, int W, int H)
{
    if (z.flowType == ALIEN_B200_FLOW_RADIAL) {
        const float baseValue = zoneFlowHeight(z, pos, W, H);
        const float downValue = zoneFlowHeight(z, pos + f2(0.0f, 1.0f), W, H);
        const float rightValue = zoneFlowHeight(z, pos + f2(1.0f, 0.0f), W, H);
        return rotateClockwiseDeg(f2(rightValue - baseValue, downValue - baseValue), 90.0f + z.flowDriftAngle);
    }
    if (z.flowType == ALIEN_B200_FLOW_CENTRAL) {
        const float2 center = seamDiff2(f2(z.posX, z.posY), pos, W, H);
        return center * (z.flowStrength / (lensq2(center) + 50.0f));
    }
    if (z.flowType == ALIEN_B200_FLOW_LINEAR) return unitVectorOfAngle(z.flowAngle) * z.flowStrength;
    return f2(0.0f, 0.0f);
}

// cudaApplyFlowFieldSettings (FlowFieldKernels.cu:48-89) with
// SpotCalculator::calcResultingFlowField (:58-78): the blended acceleration
__device__ __forceinline__ float2 flowAcceleration(const AlienPhysicsParams& p, float2 pos, int W, int H)
{
    if (p.numZones <= 0) return f2(0.0f, 0.0f);
    float baseFactor = 1.0f, sum = 0.0f;
    bool any = false;
    for (int i = 0; i < p.numZones; ++i) {
        const AlienZone& z = p.zones[i];
        if (z.flowType == ALIEN_B200_FLOW_NONE) continue;
        const float w = zoneWeight(z, zoneDelta(z, pos, W, H));
        baseFactor *= w;
        sum += 1.0f - w;
        any = true;
    }
    if (!any) return f2(0.0f, 0.0f);
    sum += baseFactor;
    float2 result = f2(0.0f, 0.0f) * baseFactor;
    for (int i = 0; i < p.numZones; ++i) {
        const AlienZone& z = p.zones[i];
        if (z.flowType == ALIEN_B200_FLOW_NONE) continue;
        const float w = zoneWeight(z, zoneDelta(z, pos, W, H));
        result = result + zoneFlowAcceleration(z, pos, W, H) * (1.0f - w) / sum;
    }
    return result;
}

__device__ __forceinline__ bool anyFlow(const AlienPhysicsParams& p)
{
    for (int i = 0; i < p.numZones; ++i)
        if (p.zones[i].flowType != ALIEN_B200_FLOW_NONE) return true;
    return false;
}

// RadiationProcessor::calcActiveSources (RadiationProcessor.cuh:42-59): bit i
// set for an active source i (its position not in a zone that disables the
// sources)
__device__ __forceinline__ unsigned long long activeSources(const AlienPhysicsParams& p, int W, int H)
{
    unsigned long long mask = 0;
    for (int i = 0; i < p.numRadiationSources; ++i) {
        const AlienRadiationSource& r = p.radiationSources[i];
        const float disabled = zoneParam<kZRadiationDisableSources>(p, W, H, f2(r.posX, r.posY),
                                                                   p.radiationDisableSources ? 1.0f : 0.0f);
        if (!(disabled > 0.5f)) mask |= 1ull << i;
    }
    return mask;
}

// draw sites of createEnergyParticle: base + 0 source choice, base + 1 + 2k
// and base + 2 + 2k the k-th try of a circular offset (k < 10), base + 21 the
// speed, base + 22 / 23 the rectangular offset
constexpr uint32_t kSiteSourceRadiation = 32;
constexpr uint32_t kSiteSourceDeletedCell = 64;

// createEnergyParticle's placement at a radiation source (:252-343); pos and
// vel are changed only when a source is matched
__device__ __forceinline__ void placeAtSource(const AlienPhysicsParams& p, unsigned long long mask, uint64_t id, uint64_t T,
                                              uint32_t site, float2& pos, float2& vel)
{
    if (mask == 0) return;
    float sumRatios = 0.0f;
    for (int i = 0; i < p.numRadiationSources; ++i)
        if ((mask >> i) & 1ull) sumRatios += p.radiationSources[i].strength;
    if (!(sumRatios > 0.0f)) return;
    const float r = draw(id, T, site);
    sumRatios = 0.0f;
    int index = -1;
    for (int i = 0; i < p.numRadiationSources; ++i) {
        if (!((mask >> i) & 1ull)) continue;
        sumRatios += p.radiationSources[i].strength;
        if (r <= sumRatios) {
            index = i;
            break;
        }
    }
    if (index < 0) return;
    const AlienRadiationSource& src = p.radiationSources[index];
    pos = f2(src.posX, src.posY);
    const float speed = 0.5f + 0.5f * draw(id, T, site + 21);
    if (src.shapeType == ALIEN_B200_SHAPE_CIRCULAR) {
        const float radius = fmaxf(1.0f, src.radius);
        float2 delta = f2(0.0f, 0.0f);
        for (int k = 0; k < 10; ++k) {
            delta.x = draw(id, T, site + 1 + 2 * k) * radius * 2.0f - radius;
            delta.y = draw(id, T, site + 2 + 2 * k) * radius * 2.0f - radius;
            if (len2(delta) <= radius) break;
        }
        pos = pos + delta;
        vel = src.useAngle ? unitVectorOfAngle(src.angle) * speed : normalized2(delta) * speed;
    } else {
        const float w = src.width, h = src.height;
        float2 delta;
        delta.x = draw(id, T, site + 22) * w - w / 2;
        delta.y = draw(id, T, site + 23) * h - h / 2;
        pos = pos + delta;
        if (src.useAngle) {
            vel = unitVectorOfAngle(src.angle) * speed;
        } else {
            const float round = fminf(w, h) / 2;
            const float2 c1 = f2(-w / 2, -h / 2), c2 = f2(w / 2, -h / 2), c3 = f2(-w / 2, h / 2), c4 = f2(w / 2, h / 2);
            auto lengthMax = [](float2 v) { return fmaxf(fabsf(v.x), fabsf(v.y)); };
            if (lengthMax(c1 - delta) <= round) {
                vel = normalized2(delta - (c1 + f2(round, round)));
            } else if (lengthMax(c2 - delta) <= round) {
                vel = normalized2(delta - (c2 + f2(-round, round)));
            } else if (lengthMax(c3 - delta) <= round) {
                vel = normalized2(delta - (c3 + f2(round, -round)));
            } else if (lengthMax(c4 - delta) <= round) {
                vel = normalized2(delta - (c4 + f2(-round, -round)));
            } else {
                vel = f2(0.0f, 0.0f);
                const float dx1 = w / 2 + delta.x, dx2 = w / 2 - delta.x, dy1 = h / 2 + delta.y, dy2 = h / 2 - delta.y;
                if (dx1 <= dy1 && dx1 <= dy2 && delta.x <= 0) vel.x = -1;
                if (dy1 <= dx1 && dy1 <= dx2 && delta.y <= 0) vel.y = -1;
                if (dx2 <= dy1 && dx2 <= dy2 && delta.x > 0) vel.x = 1;
                if (dy2 <= dx1 && dy2 <= dx2 && delta.y > 0) vel.y = 1;
            }
            vel = vel * speed;
        }
    }
}

// SimulationParametersUpdateService::updateSimulationParametersAfterTimestep
// (SimulationParametersUpdateService.cu:52-78): a source or zone whose
// velocity exceeds NEAR_ZERO moves by velocity * dt, wrapped onto the torus
__device__ __forceinline__ void moveOnTorus(float& x, float& y, float vx, float vy, float dt, int W, int H)
{
    if (fabsf(vx) > kNearZero) x += vx * dt;
    if (fabsf(vy) > kNearZero) y += vy * dt;
    const float2 c = correctPosition(f2(x, y), W, H);
    x = c.x;
    y = c.y;
}
__device__ __forceinline__ void moveZonesAndSources(AlienPhysicsParams& p, int W, int H)
{
    for (int i = 0; i < p.numRadiationSources; ++i) {
        AlienRadiationSource& r = p.radiationSources[i];
        moveOnTorus(r.posX, r.posY, r.velX, r.velY, p.timestepSize, W, H);
    }
    for (int i = 0; i < p.numZones; ++i) {
        AlienZone& z = p.zones[i];
        moveOnTorus(z.posX, z.posY, z.velX, z.velY, p.timestepSize, W, H);
    }
}

// 2^-24 fixed point of the external-energy backflow (order-independent sums)
constexpr double kBackflowScale = 16777216.0;

// the external-energy backflow of a new energy particle (:345-354): with the
// feature on and a positive backflow factor for the color, the pool takes
// energy * factor unless that would raise the pool above its limit (tested
// against the pool at the start of the step, so the outcome does not depend
// on the order of the step's particles); returns the particle's energy and
// adds the backflow to the world's step accumulator
__device__ __forceinline__ float backflow(const AlienPhysicsParams& p, WorldCounters& wc, int color, float energy)
{
    if (!p.externalEnergyControl || !(p.externalEnergyBackflowFactor[color] > 0.0f)) return energy;
    const float factor = p.externalEnergyBackflowFactor[color];
    const double add = static_cast<double>(energy * factor);
    if (wc.externalEnergy + add > static_cast<double>(p.externalEnergyBackflowLimit)) return energy;
    atomicAdd(reinterpret_cast<unsigned long long*>(&wc.backflowFix), static_cast<unsigned long long>(__double2ll_rn(add * kBackflowScale)));
    return energy * (1.0f - factor);
}

// the particle energy a backflow leaves, without recording it
__device__ __forceinline__ float backflowKept(const AlienPhysicsParams& p, const WorldCounters& wc, int color, float energy)
{
    if (!p.externalEnergyControl || !(p.externalEnergyBackflowFactor[color] > 0.0f)) return energy;
    const float factor = p.externalEnergyBackflowFactor[color];
    if (wc.externalEnergy + static_cast<double>(energy * factor) > static_cast<double>(p.externalEnergyBackflowLimit)) return energy;
    return energy * (1.0f - factor);
}

}  // namespace ab
