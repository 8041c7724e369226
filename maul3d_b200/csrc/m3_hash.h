// The world hash: FNV-1a 64 over the curated world state in canonical
// slot order, folding exactly the bytes, in exactly the order and under
// exactly the off-default conditions, of the reference's m3World_Hash
// (src/snapshot.c:932-1345).  One function serves the host (over the
// host image) and the device (one thread per world over the HBM slab).
//
// Subsystems the device path does not model (characters, soft bodies,
// vehicles, voxel chunks, water volumes) hold no live slots in a world
// this library creates; their loops fold nothing in the reference
// either (empty pools), so they are absent here.
#ifndef M3_HASH_H
#define M3_HASH_H

#include "m3_layout.h"

M3_HD uint64_t m3WorldHashView(const m3WorldView* w)
{
    const m3WorldScalars* sc = w->sc;
    uint64_t h = M3_HASH_INIT;
    h = m3Fnv(h, &sc->stepCount, 8);
    h = m3Fnv(h, &sc->gravity, 12);
    if (sc->contactHertz != M3_CONTACT_HERTZ_DEFAULT ||
        sc->contactDampingRatio != M3_CONTACT_DAMPING_RATIO_DEFAULT ||
        sc->contactPushMaxSpeed != M3_CONTACT_PUSH_MAX_SPEED_DEFAULT ||
        sc->restitutionThreshold != M3_RESTITUTION_THRESHOLD_DEFAULT ||
        sc->maximumLinearSpeed != M3_MAX_LINEAR_SPEED_DEFAULT || sc->sleepEnabled == 0 ||
        sc->continuousEnabled == 0 || sc->hitEventThreshold != M3_HIT_EVENT_THRESHOLD_DEFAULT)
    {
        h = m3Fnv(h, &sc->contactHertz, 4);
        h = m3Fnv(h, &sc->contactDampingRatio, 4);
        h = m3Fnv(h, &sc->contactPushMaxSpeed, 4);
        h = m3Fnv(h, &sc->restitutionThreshold, 4);
        h = m3Fnv(h, &sc->maximumLinearSpeed, 4);
        h = m3Fnv(h, &sc->sleepEnabled, 1);
        h = m3Fnv(h, &sc->continuousEnabled, 1);
        h = m3Fnv(h, &sc->hitEventThreshold, 4);
    }
    if (sc->maximumAngularSpeed != M3_MAX_ANGULAR_SPEED_DEFAULT)
    {
        h = m3Fnv(h, &sc->maximumAngularSpeed, 4);
    }
    if (sc->windSpeed != 0.0f)
    {
        h = m3Fnv(h, &sc->windDir, 12);
        h = m3Fnv(h, &sc->windSpeed, 4);
        h = m3Fnv(h, &sc->windGustHertz, 4);
        h = m3Fnv(h, &sc->windGustScale, 4);
        h = m3Fnv(h, &sc->windPhase, 4);
    }
    for (int32_t i = 0; i < sc->bodyMax; ++i)
    {
        uint8_t alive = w->bodyAlive[i];
        h = m3Fnv(h, &alive, 1);
        if (alive == 0)
        {
            continue;
        }
        h = m3Fnv(h, &w->xf[i], 40);
        h = m3Fnv(h, &w->v[i], 12);
        m3Vec3 f = w->force[i];
        m3Vec3 t = w->torque[i];
        if (f.x != 0.0f || f.y != 0.0f || f.z != 0.0f || t.x != 0.0f || t.y != 0.0f ||
            t.z != 0.0f)
        {
            h = m3Fnv(h, &w->force[i], 12);
            h = m3Fnv(h, &w->torque[i], 12);
        }
        if (w->enabled[i] == 0 || w->locks[i] != 0 ||
            w->sleepThreshold[i] != M3_SLEEP_VELOCITY_DEFAULT || w->canSleep[i] == 0 ||
            w->hasTarget[i] != 0)
        {
            h = m3Fnv(h, &w->enabled[i], 1);
            h = m3Fnv(h, &w->locks[i], 1);
            h = m3Fnv(h, &w->sleepThreshold[i], 4);
            h = m3Fnv(h, &w->canSleep[i], 1);
            h = m3Fnv(h, &w->hasTarget[i], 1);
            h = m3Fnv(h, &w->target[i], 40);
        }
        h = m3Fnv(h, &w->w[i], 12);
        h = m3Fnv(h, &w->invMass[i], 4);
        h = m3Fnv(h, &w->invI[i], 36);
        h = m3Fnv(h, &w->lc[i], 12);
        h = m3Fnv(h, &w->btype[i], 1);
        h = m3Fnv(h, &w->bullet[i], 1);
        h = m3Fnv(h, &w->awake[i], 1);
        h = m3Fnv(h, &w->sleepTime[i], 4);
    }
    const int32_t minusOne = -1;
    for (int32_t i = 0; i < sc->shapeMax; ++i)
    {
        uint8_t alive = w->shapeAlive[i];
        h = m3Fnv(h, &alive, 1);
        if (alive == 0)
        {
            continue;
        }
        h = m3Fnv(h, &w->shapeBody[i], 4);
        h = m3Fnv(h, &w->shapeType[i], 1);
        h = m3Fnv(h, &w->geom[i], 32);
        h = m3Fnv(h, &w->density[i], 4);
        h = m3Fnv(h, &w->friction[i], 4);
        h = m3Fnv(h, &w->restitution[i], 4);
        if (w->hitEvents[i] != 0 || w->preSolve[i] != 0)
        {
            h = m3Fnv(h, &w->hitEvents[i], 1);
            h = m3Fnv(h, &w->preSolve[i], 1);
        }
        m3Vec3 sv = w->surfVel[i];
        if (sv.x != 0.0f || sv.y != 0.0f || sv.z != 0.0f)
        {
            h = m3Fnv(h, &w->surfVel[i], 12);
        }
        if (w->hasOffset[i] != 0)
        {
            h = m3Fnv(h, &w->localPos[i], 12);
            h = m3Fnv(h, &w->localRot[i], 16);
        }
        if (w->rolling[i] != 0.0f)
        {
            h = m3Fnv(h, &w->rolling[i], 4);
        }
        if (w->category[i] != 1ull || w->mask[i] != ~0ull || w->group[i] != 0)
        {
            h = m3Fnv(h, &w->category[i], 8);
            h = m3Fnv(h, &w->mask[i], 8);
            h = m3Fnv(h, &w->group[i], 4);
        }
        h = m3Fnv(h, &w->hullIndex[i], 4);
        h = m3Fnv(h, &minusOne, 4); // mesh slot: no mesh shapes on this path
        h = m3Fnv(h, &w->sensor[i], 1);
    }
    for (int32_t i = 0; i < sc->jointMax; ++i)
    {
        uint8_t alive = w->jointAlive[i];
        h = m3Fnv(h, &alive, 1);
        if (alive == 0)
        {
            continue;
        }
        h = m3Fnv(h, &w->jtype[i], 1);
        h = m3Fnv(h, &w->jbodyA[i], 4);
        h = m3Fnv(h, &w->jbodyB[i], 4);
        h = m3Fnv(h, &w->jlocalA[i], 12);
        h = m3Fnv(h, &w->jlocalB[i], 12);
        h = m3Fnv(h, &w->jimpulse[i], 12);
        if (w->jbreak[i].x != 0.0f || w->jbreak[i].y != 0.0f)
        {
            h = m3Fnv(h, &w->jbreak[i], 12);
        }
        m3Quat tq = w->jtargetQ[i];
        m3Vec3 si = w->jspringImp[i];
        if ((w->jflags[i] & 8) != 0 || w->jtargetScalar[i] != 0.0f || tq.x != 0.0f ||
            tq.y != 0.0f || tq.z != 0.0f || tq.w != 1.0f || si.x != 0.0f || si.y != 0.0f ||
            si.z != 0.0f)
        {
            h = m3Fnv(h, &w->jspring[i], 12);
            h = m3Fnv(h, &w->jtargetScalar[i], 4);
            h = m3Fnv(h, &w->jtargetQ[i], 16);
            h = m3Fnv(h, &w->jspringImp[i], 12);
        }
        h = m3Fnv(h, &w->jperp[i], 12);
        h = m3Fnv(h, &w->jlimitImp[i], 12);
        h = m3Fnv(h, &w->jangular[i], 12);
        h = m3Fnv(h, &w->jframeA[i], 16);
        h = m3Fnv(h, &w->jframeB[i], 16);
        h = m3Fnv(h, &w->jflags[i], 1);
    }
    int32_t pairCount = sc->pairCount;
    h = m3Fnv(h, &pairCount, 4);
    const uint64_t* keys = sc->pairBuf == 0 ? w->keys0 : w->keys1;
    const m3Manifold* man = sc->pairBuf == 0 ? w->man0 : w->man1;
    for (int32_t i = 0; i < pairCount; ++i)
    {
        h = m3Fnv(h, &keys[i], 8);
        h = m3Fnv(h, &man[i], 188);
    }
    return h;
}

#endif // M3_HASH_H
