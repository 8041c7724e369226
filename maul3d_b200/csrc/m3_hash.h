// The world hash: FNV-1a 64 over the curated world state in canonical
// slot order, folding exactly the bytes, in exactly the order and under
// exactly the off-default conditions, of the reference's m3World_Hash
// (src/snapshot.c:932-1345).
//
// The byte stream is defined once, as a sequence of records (the world
// header, one record per body slot, per shape slot, per joint slot, the
// pair count, one record per current pair), each emitted into a sink:
// an FNV folder (the host hash and the reference-order definition), a
// byte counter, or the device kernel's shared-memory stager, which
// hashes the same stream in parallel.
//
// Subsystems the device path does not model (characters, soft bodies,
// vehicles, voxel chunks, water volumes) hold no live slots in a world
// this library creates; their loops fold nothing in the reference
// either (empty pools), so they are absent here.
#ifndef M3_HASH_H
#define M3_HASH_H

#include "m3_layout.h"

struct m3FnvSink
{
    uint64_t h;
    M3_HD_MEMBER void put(const void* p, int32_t n)
    {
        h = m3Fnv(h, p, n);
    }
};

struct m3CountSink
{
    int32_t n;
    M3_HD_MEMBER void put(const void*, int32_t k)
    {
        n += k;
    }
};

// snapshot.c:932-960: step count, gravity, the tuning block when any
// knob is off its default, the angular cap, the wind block.
template <class Sink> M3_HD void m3HashHeader(const m3WorldView* w, Sink& k)
{
    const m3WorldScalars* sc = w->sc;
    k.put(&sc->stepCount, 8);
    k.put(&sc->gravity, 12);
    if (sc->contactHertz != M3_CONTACT_HERTZ_DEFAULT ||
        sc->contactDampingRatio != M3_CONTACT_DAMPING_RATIO_DEFAULT ||
        sc->contactPushMaxSpeed != M3_CONTACT_PUSH_MAX_SPEED_DEFAULT ||
        sc->restitutionThreshold != M3_RESTITUTION_THRESHOLD_DEFAULT ||
        sc->maximumLinearSpeed != M3_MAX_LINEAR_SPEED_DEFAULT || sc->sleepEnabled == 0 ||
        sc->continuousEnabled == 0 || sc->hitEventThreshold != M3_HIT_EVENT_THRESHOLD_DEFAULT)
    {
        k.put(&sc->contactHertz, 4);
        k.put(&sc->contactDampingRatio, 4);
        k.put(&sc->contactPushMaxSpeed, 4);
        k.put(&sc->restitutionThreshold, 4);
        k.put(&sc->maximumLinearSpeed, 4);
        k.put(&sc->sleepEnabled, 1);
        k.put(&sc->continuousEnabled, 1);
        k.put(&sc->hitEventThreshold, 4);
    }
    if (sc->maximumAngularSpeed != M3_MAX_ANGULAR_SPEED_DEFAULT)
    {
        k.put(&sc->maximumAngularSpeed, 4);
    }
    if (sc->windSpeed != 0.0f)
    {
        k.put(&sc->windDir, 12);
        k.put(&sc->windSpeed, 4);
        k.put(&sc->windGustHertz, 4);
        k.put(&sc->windGustScale, 4);
        k.put(&sc->windPhase, 4);
    }
}

// One body slot: the alive byte, then the body state when alive.
template <class Sink> M3_HD void m3HashBody(const m3WorldView* w, int32_t i, Sink& k)
{
    const uint8_t alive = w->bodyAlive[i];
    k.put(&alive, 1);
    if (alive == 0)
    {
        return;
    }
    k.put(&w->xf[i], 40);
    k.put(&w->v[i], 12);
    const m3Vec3 f = w->force[i];
    const m3Vec3 t = w->torque[i];
    if (f.x != 0.0f || f.y != 0.0f || f.z != 0.0f || t.x != 0.0f || t.y != 0.0f || t.z != 0.0f)
    {
        k.put(&w->force[i], 12);
        k.put(&w->torque[i], 12);
    }
    if (w->enabled[i] == 0 || w->locks[i] != 0 ||
        w->sleepThreshold[i] != M3_SLEEP_VELOCITY_DEFAULT || w->canSleep[i] == 0 ||
        w->hasTarget[i] != 0)
    {
        k.put(&w->enabled[i], 1);
        k.put(&w->locks[i], 1);
        k.put(&w->sleepThreshold[i], 4);
        k.put(&w->canSleep[i], 1);
        k.put(&w->hasTarget[i], 1);
        k.put(&w->target[i], 40);
    }
    k.put(&w->w[i], 12);
    k.put(&w->invMass[i], 4);
    k.put(&w->invI[i], 36);
    k.put(&w->lc[i], 12);
    k.put(&w->btype[i], 1);
    k.put(&w->bullet[i], 1);
    k.put(&w->awake[i], 1);
    k.put(&w->sleepTime[i], 4);
}

// One shape slot.
template <class Sink> M3_HD void m3HashShape(const m3WorldView* w, int32_t i, Sink& k)
{
    const uint8_t alive = w->shapeAlive[i];
    k.put(&alive, 1);
    if (alive == 0)
    {
        return;
    }
    k.put(&w->shapeBody[i], 4);
    k.put(&w->shapeType[i], 1);
    k.put(&w->geom[i], 32);
    k.put(&w->density[i], 4);
    k.put(&w->friction[i], 4);
    k.put(&w->restitution[i], 4);
    if (w->hitEvents[i] != 0 || w->preSolve[i] != 0)
    {
        k.put(&w->hitEvents[i], 1);
        k.put(&w->preSolve[i], 1);
    }
    const m3Vec3 sv = w->surfVel[i];
    if (sv.x != 0.0f || sv.y != 0.0f || sv.z != 0.0f)
    {
        k.put(&w->surfVel[i], 12);
    }
    if (w->hasOffset[i] != 0)
    {
        k.put(&w->localPos[i], 12);
        k.put(&w->localRot[i], 16);
    }
    if (w->rolling[i] != 0.0f)
    {
        k.put(&w->rolling[i], 4);
    }
    if (w->category[i] != 1ull || w->mask[i] != ~0ull || w->group[i] != 0)
    {
        k.put(&w->category[i], 8);
        k.put(&w->mask[i], 8);
        k.put(&w->group[i], 4);
    }
    k.put(&w->hullIndex[i], 4);
    const int32_t minusOne = -1; // mesh slot: no mesh shapes on this path
    k.put(&minusOne, 4);
    k.put(&w->sensor[i], 1);
}

// One joint slot.
template <class Sink> M3_HD void m3HashJoint(const m3WorldView* w, int32_t i, Sink& k)
{
    const uint8_t alive = w->jointAlive[i];
    k.put(&alive, 1);
    if (alive == 0)
    {
        return;
    }
    k.put(&w->jtype[i], 1);
    k.put(&w->jbodyA[i], 4);
    k.put(&w->jbodyB[i], 4);
    k.put(&w->jlocalA[i], 12);
    k.put(&w->jlocalB[i], 12);
    k.put(&w->jimpulse[i], 12);
    if (w->jbreak[i].x != 0.0f || w->jbreak[i].y != 0.0f)
    {
        k.put(&w->jbreak[i], 12);
    }
    const m3Quat tq = w->jtargetQ[i];
    const m3Vec3 si = w->jspringImp[i];
    if ((w->jflags[i] & 8) != 0 || w->jtargetScalar[i] != 0.0f || tq.x != 0.0f || tq.y != 0.0f ||
        tq.z != 0.0f || tq.w != 1.0f || si.x != 0.0f || si.y != 0.0f || si.z != 0.0f)
    {
        k.put(&w->jspring[i], 12);
        k.put(&w->jtargetScalar[i], 4);
        k.put(&w->jtargetQ[i], 16);
        k.put(&w->jspringImp[i], 12);
    }
    k.put(&w->jperp[i], 12);
    k.put(&w->jlimitImp[i], 12);
    k.put(&w->jangular[i], 12);
    k.put(&w->jframeA[i], 16);
    k.put(&w->jframeB[i], 16);
    k.put(&w->jflags[i], 1);
}

// One current pair: its key and its manifold.
template <class Sink> M3_HD void m3HashPair(const m3WorldView* w, int32_t i, Sink& k)
{
    const uint64_t* keys = w->sc->pairBuf == 0 ? w->keys0 : w->keys1;
    const m3Manifold* man = w->sc->pairBuf == 0 ? w->man0 : w->man1;
    k.put(&keys[i], 8);
    k.put(&man[i], 188);
}

// Records of the stream: header, bodies, shapes, joints, pair count,
// pairs.
M3_HD int32_t m3HashRecordCount(const m3WorldView* w)
{
    const m3WorldScalars* sc = w->sc;
    return 2 + sc->bodyMax + sc->shapeMax + sc->jointMax + sc->pairCount;
}

template <class Sink> M3_HD void m3HashRecord(const m3WorldView* w, int32_t r, Sink& k)
{
    const m3WorldScalars* sc = w->sc;
    if (r == 0)
    {
        m3HashHeader(w, k);
        return;
    }
    r -= 1;
    if (r < sc->bodyMax)
    {
        m3HashBody(w, r, k);
        return;
    }
    r -= sc->bodyMax;
    if (r < sc->shapeMax)
    {
        m3HashShape(w, r, k);
        return;
    }
    r -= sc->shapeMax;
    if (r < sc->jointMax)
    {
        m3HashJoint(w, r, k);
        return;
    }
    r -= sc->jointMax;
    if (r == 0)
    {
        k.put(&sc->pairCount, 4);
        return;
    }
    m3HashPair(w, r - 1, k);
}

// The whole stream folded sequentially (the host path and the
// definition the parallel device hash is tested against).
M3_HD uint64_t m3WorldHashView(const m3WorldView* w)
{
    m3FnvSink k{M3_HASH_INIT};
    const int32_t n = m3HashRecordCount(w);
    for (int32_t r = 0; r < n; ++r)
    {
        m3HashRecord(w, r, k);
    }
    return k.h;
}

#endif // M3_HASH_H
