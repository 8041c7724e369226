// Seeded synthetic scenes: the workload generator for tests and the
// benchmark.  Written against the reference-named public API only, so
// the very same source builds a world in this library and, compiled
// against the reference's headers (oracle/Makefile), in the reference
// engine.  Both worlds then hold identical bytes from identical seeds.
//
// Randomness is SplitMix64 (Steele, Lea, Flood 2014), the generator
// the reference bench uses for its scenes (bench/bench_main.c:44-57),
// mapped to [lo, hi) through the top 53 bits.
//
// Scenes:
//   M3S_SPHERE_PYRAMID  the reference bench "pyramid" layout
//                       (bench/bench_main.c:68-96); its hash after 300
//                       steps of dt 1/60, 4 substeps is pinned in
//                       bench/pins.txt:1 (975f319f2f44cc5d).
//   M3S_BOX_PYRAMID     a 2D wall pyramid of unit boxes on a plane,
//                       `param` rows (20 rows = 210 boxes).
//   M3S_UNEVEN          one world of the batched workload: `param`
//                       dynamic bodies of 8-high box stacks, loose
//                       spheres and three revolute chains of 8 capsules
//                       hung from static anchors, laid out from `seed`.
//   M3S_FREEFALL        `param` spheres and boxes in free fall, no
//                       contacts for the first steps (integration only).
//   M3S_TOWERS          `param` towers of 2x2x4 unit boxes welded to
//                       their face neighbours by breakable fixed joints
//                       (28 a tower), each hit by a sphere launched at
//                       20-40 m/s: joints break on impact and their
//                       slots are recycled.
//   M3S_TERRAIN         `param` spheres, capsules and boxes dropped a
//                       short way onto a seeded heightfield (1 m cells,
//                       a sum of three sine waves, about 0.6 m high),
//                       the heightfield versus convex contacts.
//   M3S_SHOTS           `param` small spheres, boxes and capsules shot at
//                       25-60 m/s across a ring of static boxes, spheres
//                       and capsules above a ground plane (odd seeds add
//                       a heightfield patch): the continuous phase's time
//                       of impact against static targets.
//   M3S_PLANK           `param` small boxes (at least 17) resting on one
//                       dynamic plank on the ground: the plank carries
//                       more constraints than there are graph colours,
//                       so the solver's overflow colour is used.
//   M3S_BOUNCE          `param` spheres and boxes with restitution 0.3-0.8
//                       dropped from 2-8 m onto a bouncy ground and onto
//                       each other: the restitution pass.
//   M3S_CITY            the large single world: `param` towers of
//                       10 x 10 x 2 unit boxes (10 wide, 10 high, 2 deep)
//                       welded to their six neighbours by fixed joints
//                       that break at 500 N (460 joints a tower), on a
//                       grid 16 m apart, and four spheres (radius 0.5)
//                       per tower launched at 20-40 m/s toward seeded
//                       towers: 1000 towers are 204,000 bodies and
//                       460,000 joints.
//   M3S_RAIN            the mixed rain field: `param` bodies (10,000 in
//                       the configuration), 40 % spheres, 30 % capsules,
//                       30 % QuickHull hulls of 16-32 points, on a jittered
//                       grid 2.4 m apart at heights 5-100 m above a
//                       255 x 255 heightfield of 1 m cells (four seeded
//                       sine octaves, 4 m amplitude).
//   M3S_MIXED           one served world: `param` dynamic bodies, a third
//                       each boxes (half extent U[0.25, 0.5]), spheres
//                       (radius U[0.25, 0.5]) and QuickHull hulls of 16
//                       points on a sphere of radius U[0.3, 0.6], in
//                       columns of four on a jittered 1.6 m grid above a
//                       ground plane, dropped from 0.1-0.4 m gaps.

#include <m3_scene_api.h> // resolved by -I: product or oracle shim

#include <math.h>
#include <stdint.h>

enum
{
    M3S_SPHERE_PYRAMID = 0,
    M3S_BOX_PYRAMID = 1,
    M3S_UNEVEN = 2,
    M3S_FREEFALL = 3,
    M3S_TOWERS = 4,
    M3S_TERRAIN = 5,
    M3S_SHOTS = 6,
    M3S_PLANK = 7,
    M3S_BOUNCE = 8,
    M3S_CITY = 9,
    M3S_RAIN = 10,
    M3S_MIXED = 11,
};

static uint64_t SceneSplitMix(uint64_t* state)
{
    *state += 0x9E3779B97F4A7C15ull;
    uint64_t z = *state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double SceneRand(uint64_t* state, double lo, double hi)
{
    double unit = (double)(SceneSplitMix(state) >> 11) * (1.0 / 9007199254740992.0);
    return lo + (hi - lo) * unit;
}

static m3BodyId SceneGround(m3WorldId world, float friction)
{
    m3BodyDef gd = m3DefaultBodyDef();
    m3BodyId ground = m3CreateBody(world, &gd);
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = friction;
    m3Plane floor = {{0.0f, 1.0f, 0.0f}, 0.0f};
    m3CreatePlaneShape(ground, &sd, &floor);
    return ground;
}

static m3WorldId SphereLayers(void)
{
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = 256;
    def.shapeCapacity = 256;
    m3WorldId world = m3CreateWorld(&def);
    SceneGround(world, 0.6f);
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = 0.6f;
    for (int32_t layer = 0; layer < 6; ++layer)
    {
        int32_t n = 6 - layer;
        for (int32_t i = 0; i < n; ++i)
        {
            for (int32_t j = 0; j < n; ++j)
            {
                bd.position = (m3Pos3){(double)i - 0.5 * (double)n + 0.05 * (double)layer,
                                       0.5 + 1.02 * (double)layer, (double)j - 0.5 * (double)n};
                m3BodyId body = m3CreateBody(world, &bd);
                m3Sphere ball = {{0.0f, 0.0f, 0.0f}, 0.5f};
                m3CreateSphereShape(body, &sd, &ball);
            }
        }
    }
    return world;
}

static m3WorldId BoxWall(int32_t rows)
{
    m3WorldDef def = m3DefaultWorldDef();
    m3WorldId world = m3CreateWorld(&def);
    SceneGround(world, 0.6f);
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = 0.6f;
    sd.density = 1.0f;
    for (int32_t r = 0; r < rows; ++r)
    {
        int32_t n = rows - r;
        for (int32_t i = 0; i < n; ++i)
        {
            bd.position =
                (m3Pos3){(double)i - 0.5 * (double)n + 0.5, 0.5 + (double)r, 0.0};
            m3BodyId body = m3CreateBody(world, &bd);
            m3CreateBoxShape(body, &sd, (m3Vec3){0.5f, 0.5f, 0.5f});
        }
    }
    return world;
}

static m3WorldId UnevenWorld(uint64_t seed, int32_t bodies)
{
    if (bodies < 32)
    {
        bodies = 32;
    }
    const int32_t chainCount = 3;
    const int32_t chainLinks = 8;
    int32_t rest = bodies - chainCount * chainLinks;
    int32_t stacks = (rest * 2 / 3) / 8;
    int32_t spheres = rest - 8 * stacks;

    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = bodies + 8;
    def.shapeCapacity = bodies + 8;
    def.jointCapacity = chainCount * chainLinks + 8;
    m3WorldId world = m3CreateWorld(&def);
    SceneGround(world, 0.6f);

    uint64_t rng = seed;
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = 0.6f;
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;

    // Box stacks on a square grid of 2.5 m cells, one half extent per
    // stack drawn from U[0.25, 0.75], boxes resting face to face.
    int32_t side = 1;
    while (side * side < stacks + spheres / 4 + 4)
    {
        side += 1;
    }
    for (int32_t s = 0; s < stacks; ++s)
    {
        double cx = 2.5 * (double)(s % side) - 1.25 * (double)side;
        double cz = 2.5 * (double)(s / side) - 1.25 * (double)side;
        float h = (float)SceneRand(&rng, 0.25, 0.75);
        for (int32_t k = 0; k < 8; ++k)
        {
            bd.position = (m3Pos3){cx, (double)h * (double)(2 * k + 1), cz};
            bd.linearVelocity = (m3Vec3){0.0f, 0.0f, 0.0f};
            m3BodyId body = m3CreateBody(world, &bd);
            m3CreateBoxShape(body, &sd, (m3Vec3){h, h, h});
        }
    }

    // Loose spheres thrown low across the field: radius U[0.2, 0.5],
    // a short drop and a horizontal velocity toward the stacks.
    for (int32_t b = 0; b < spheres; ++b)
    {
        float r = (float)SceneRand(&rng, 0.2, 0.5);
        double x = -1.25 * (double)side + 1.2 * (double)(b / 16);
        double z = -1.25 * (double)side - 3.0 - 1.2 * (double)(b % 16);
        bd.position = (m3Pos3){x, (double)r + SceneRand(&rng, 0.0, 0.3), z};
        bd.linearVelocity = (m3Vec3){(float)SceneRand(&rng, -1.0, 1.0), 0.0f,
                                     (float)SceneRand(&rng, 1.0, 3.0)};
        m3BodyId body = m3CreateBody(world, &bd);
        m3Sphere ball = {{0.0f, 0.0f, 0.0f}, r};
        m3CreateSphereShape(body, &sd, &ball);
    }
    bd.linearVelocity = (m3Vec3){0.0f, 0.0f, 0.0f};

    // Three revolute chains: a shapeless static anchor, 8 capsule
    // links (radius 0.1, half-height 0.4) laid out horizontally from
    // it along +x, hinged about z, released to swing down.
    for (int32_t c = 0; c < chainCount; ++c)
    {
        double ax = 1.25 * (double)side + 1.0;
        double ay = 9.5;
        double az = -1.25 * (double)side + 2.5 * (double)c;
        m3BodyDef anchorDef = m3DefaultBodyDef();
        anchorDef.position = (m3Pos3){ax, ay, az};
        m3BodyId prev = m3CreateBody(world, &anchorDef);
        for (int32_t k = 0; k < chainLinks; ++k)
        {
            bd.position = (m3Pos3){ax + 0.5 + 1.0 * (double)k, ay, az};
            m3BodyId link = m3CreateBody(world, &bd);
            m3Capsule cap = {{-0.4f, 0.0f, 0.0f}, {0.4f, 0.0f, 0.0f}, 0.1f};
            m3CreateCapsuleShape(link, &sd, &cap);
            m3JointDef jd = m3DefaultJointDef();
            jd.type = m3_revoluteJoint;
            jd.bodyA = prev;
            jd.bodyB = link;
            jd.localAnchorA = k == 0 ? (m3Vec3){0.0f, 0.0f, 0.0f} : (m3Vec3){0.5f, 0.0f, 0.0f};
            jd.localAnchorB = (m3Vec3){-0.5f, 0.0f, 0.0f};
            jd.localAxisA = (m3Vec3){0.0f, 0.0f, 1.0f};
            jd.localAxisB = (m3Vec3){0.0f, 0.0f, 1.0f};
            m3CreateJoint(&jd);
            prev = link;
        }
    }
    return world;
}

static m3WorldId FreeFall(int32_t count)
{
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = count + 4;
    def.shapeCapacity = count + 4;
    m3WorldId world = m3CreateWorld(&def);
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    m3ShapeDef sd = m3DefaultShapeDef();
    uint64_t rng = 0xF4EEull;
    for (int32_t k = 0; k < count; ++k)
    {
        bd.position = (m3Pos3){3.0 * (double)k, 50.0 + SceneRand(&rng, 0.0, 5.0), 0.0};
        bd.linearVelocity = (m3Vec3){(float)SceneRand(&rng, -1.0, 1.0), 0.0f,
                                     (float)SceneRand(&rng, -1.0, 1.0)};
        bd.angularVelocity = (m3Vec3){(float)SceneRand(&rng, -2.0, 2.0),
                                      (float)SceneRand(&rng, -2.0, 2.0),
                                      (float)SceneRand(&rng, -2.0, 2.0)};
        m3BodyId body = m3CreateBody(world, &bd);
        if (k % 2 == 0)
        {
            m3Sphere ball = {{0.0f, 0.0f, 0.0f}, 0.4f};
            m3CreateSphereShape(body, &sd, &ball);
        }
        else
        {
            m3CreateBoxShape(body, &sd, (m3Vec3){0.3f, 0.45f, 0.6f});
        }
    }
    return world;
}

// Towers of 2x2x4 unit boxes 6 m apart along x.  Each box is welded to
// its +x, +y and +z neighbours by a fixed joint with a 500 N force
// threshold; every third joint also gets a 150 N*m torque threshold.  A
// dense sphere (radius 0.5, density 40) starts 8 m before each tower,
// 1-3.5 m up, flying at it at 20-40 m/s.
static m3WorldId Towers(uint64_t seed, int32_t towers)
{
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = 17 * towers + 4;
    def.shapeCapacity = 17 * towers + 4;
    def.jointCapacity = 28 * towers + 4;
    m3WorldId world = m3CreateWorld(&def);
    SceneGround(world, 0.6f);
    uint64_t rng = seed ^ 0x70BE125ull;
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = 0.6f;
    int32_t jointCount = 0;
    for (int32_t t = 0; t < towers; ++t)
    {
        double cx = 6.0 * (double)t;
        m3BodyId box[4][2][2];
        for (int32_t k = 0; k < 4; ++k)
        {
            for (int32_t j = 0; j < 2; ++j)
            {
                for (int32_t i = 0; i < 2; ++i)
                {
                    bd.position = (m3Pos3){cx + (double)i - 0.5, 0.5 + (double)k, (double)j - 0.5};
                    box[k][j][i] = m3CreateBody(world, &bd);
                    m3CreateBoxShape(box[k][j][i], &sd, (m3Vec3){0.5f, 0.5f, 0.5f});
                }
            }
        }
        for (int32_t k = 0; k < 4; ++k)
        {
            for (int32_t j = 0; j < 2; ++j)
            {
                for (int32_t i = 0; i < 2; ++i)
                {
                    for (int32_t axis = 0; axis < 3; ++axis)
                    {
                        int32_t ni = i + (axis == 0 ? 1 : 0);
                        int32_t nk = k + (axis == 1 ? 1 : 0);
                        int32_t nj = j + (axis == 2 ? 1 : 0);
                        if (ni > 1 || nk > 3 || nj > 1)
                        {
                            continue;
                        }
                        m3Vec3 half = {axis == 0 ? 0.5f : 0.0f, axis == 1 ? 0.5f : 0.0f,
                                       axis == 2 ? 0.5f : 0.0f};
                        m3JointDef jd = m3DefaultJointDef();
                        jd.type = m3_fixedJoint;
                        jd.bodyA = box[k][j][i];
                        jd.bodyB = box[nk][nj][ni];
                        jd.localAnchorA = half;
                        jd.localAnchorB = (m3Vec3){-half.x, -half.y, -half.z};
                        m3JointId joint = m3CreateJoint(&jd);
                        m3Joint_SetBreakThresholds(joint, 500.0f,
                                                   jointCount % 3 == 0 ? 150.0f : 0.0f);
                        jointCount += 1;
                    }
                }
            }
        }
        bd.position = (m3Pos3){cx - 8.0, SceneRand(&rng, 1.0, 3.5), SceneRand(&rng, -0.5, 0.5)};
        bd.linearVelocity = (m3Vec3){(float)SceneRand(&rng, 20.0, 40.0),
                                     (float)SceneRand(&rng, 0.0, 2.0), 0.0f};
        m3BodyId ball = m3CreateBody(world, &bd);
        m3Sphere shape = {{0.0f, 0.0f, 0.0f}, 0.5f};
        m3ShapeDef heavy = sd;
        heavy.density = 40.0f;
        m3CreateSphereShape(ball, &heavy, &shape);
        bd.linearVelocity = (m3Vec3){0.0f, 0.0f, 0.0f};
    }
    return world;
}

// Terrain height at (x, z) from six seeded phases.
static double TerrainWave(const double* ph, double x, double z)
{
    return 0.3 * sin(0.45 * x + ph[0]) * cos(0.38 * z + ph[1]) +
           0.18 * sin(0.83 * (x + z) + ph[2]) + 0.12 * cos(1.31 * x - 0.97 * z + ph[3]);
}

static m3WorldId Terrain(uint64_t seed, int32_t bodies)
{
    if (bodies < 3)
    {
        bodies = 3;
    }
    int32_t side = 1;
    while (side * side < bodies)
    {
        side += 1;
    }
    const float cell = 1.0f;
    int32_t n = (int32_t)(1.6 * (double)side) + 7;
    n = n > 255 ? 255 : n;
    const double half = 0.5 * (double)(n - 1) * (double)cell;

    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = bodies + 4;
    def.shapeCapacity = bodies + 4;
    def.jointCapacity = 4;
    m3WorldId world = m3CreateWorld(&def);

    uint64_t rng = seed;
    double ph[4];
    for (int32_t k = 0; k < 4; ++k)
    {
        ph[k] = SceneRand(&rng, 0.0, 6.283185307179586);
    }
    static float heights[255 * 255];
    for (int32_t iz = 0; iz < n; ++iz)
    {
        for (int32_t ix = 0; ix < n; ++ix)
        {
            heights[iz * n + ix] = (float)TerrainWave(ph, (double)ix, (double)iz);
        }
    }
    m3BodyDef gd = m3DefaultBodyDef();
    gd.position = (m3Pos3){-half, 0.0, -half};
    m3BodyId ground = m3CreateBody(world, &gd);
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = 0.6f;
    m3CreateHeightFieldGridShape(ground, &sd, heights, n, n, cell);

    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    for (int32_t b = 0; b < bodies; ++b)
    {
        // Grid coordinates in the heightfield's frame, jittered.
        double gx = 3.0 + 1.6 * (double)(b % side) + SceneRand(&rng, -0.3, 0.3);
        double gz = 3.0 + 1.6 * (double)(b / side) + SceneRand(&rng, -0.3, 0.3);
        // The highest sample of the cells around keeps the start clear.
        float top = -1.0e30f;
        for (int32_t dz = -1; dz <= 2; ++dz)
        {
            for (int32_t dx = -1; dx <= 2; ++dx)
            {
                int32_t ix = (int32_t)gx + dx;
                int32_t iz = (int32_t)gz + dz;
                ix = ix < 0 ? 0 : (ix > n - 1 ? n - 1 : ix);
                iz = iz < 0 ? 0 : (iz > n - 1 ? n - 1 : iz);
                top = heights[iz * n + ix] > top ? heights[iz * n + ix] : top;
            }
        }
        double drop = SceneRand(&rng, 0.02, 0.15);
        int32_t kind = b % 3;
        double lift;
        if (kind == 0)
        {
            float r = (float)SceneRand(&rng, 0.3, 0.5);
            lift = (double)r;
            bd.position = (m3Pos3){gx - half, (double)top + lift + drop, gz - half};
            m3BodyId body = m3CreateBody(world, &bd);
            m3Sphere ball = {{0.0f, 0.0f, 0.0f}, r};
            m3CreateSphereShape(body, &sd, &ball);
        }
        else if (kind == 1)
        {
            float r = (float)SceneRand(&rng, 0.25, 0.35);
            float hh = (float)SceneRand(&rng, 0.2, 0.45);
            lift = (double)r;
            bd.position = (m3Pos3){gx - half, (double)top + lift + drop, gz - half};
            m3BodyId body = m3CreateBody(world, &bd);
            m3Capsule cap = {{-hh, 0.0f, 0.0f}, {hh, 0.0f, 0.0f}, r};
            m3CreateCapsuleShape(body, &sd, &cap);
        }
        else
        {
            m3Vec3 he = {(float)SceneRand(&rng, 0.3, 0.45), (float)SceneRand(&rng, 0.3, 0.45),
                         (float)SceneRand(&rng, 0.3, 0.45)};
            lift = (double)he.y;
            bd.position = (m3Pos3){gx - half, (double)top + lift + drop, gz - half};
            m3BodyId body = m3CreateBody(world, &bd);
            m3CreateBoxShape(body, &sd, he);
        }
    }
    return world;
}

static m3WorldId Shots(uint64_t seed, int32_t shots)
{
    if (shots < 1)
    {
        shots = 1;
    }
    int32_t targets = shots / 3 < 4 ? 4 : shots / 3;
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = shots + targets + 4;
    def.shapeCapacity = shots + targets + 4;
    def.jointCapacity = 4;
    m3WorldId world = m3CreateWorld(&def);
    SceneGround(world, 0.6f);
    uint64_t rng = seed;
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = 0.6f;
    if ((seed & 1u) != 0)
    {
        static float patch[12 * 12];
        for (int32_t k = 0; k < 12 * 12; ++k)
        {
            patch[k] = (float)SceneRand(&rng, 0.0, 0.4);
        }
        m3BodyDef pd = m3DefaultBodyDef();
        pd.position = (m3Pos3){-5.5, 0.05, -5.5};
        m3BodyId pb = m3CreateBody(world, &pd);
        m3CreateHeightFieldGridShape(pb, &sd, patch, 12, 12, 1.0f);
    }

    // Static targets on a ring of radius 12 (a ring's width apart).
    const double ring = 12.0 + 0.5 * (double)targets;
    double tx[4096];
    double ty[4096];
    double tz[4096];
    targets = targets > 4096 ? 4096 : targets;
    m3BodyDef td = m3DefaultBodyDef();
    for (int32_t t = 0; t < targets; ++t)
    {
        double a = 6.283185307179586 * (double)t / (double)targets;
        tx[t] = ring * cos(a);
        tz[t] = ring * sin(a);
        ty[t] = SceneRand(&rng, 1.5, 3.0);
        td.position = (m3Pos3){tx[t], ty[t], tz[t]};
        m3BodyId body = m3CreateBody(world, &td);
        int32_t kind = t % 3;
        if (kind == 0)
        {
            float h = (float)SceneRand(&rng, 0.6, 1.2);
            m3CreateBoxShape(body, &sd, (m3Vec3){h, h, h});
        }
        else if (kind == 1)
        {
            m3Sphere ball = {{0.0f, 0.0f, 0.0f}, (float)SceneRand(&rng, 0.6, 1.2)};
            m3CreateSphereShape(body, &sd, &ball);
        }
        else
        {
            float hh = (float)SceneRand(&rng, 0.5, 1.0);
            m3Capsule cap = {{0.0f, -hh, 0.0f}, {0.0f, hh, 0.0f}, (float)SceneRand(&rng, 0.4, 0.7)};
            m3CreateCapsuleShape(body, &sd, &cap);
        }
    }

    // Projectiles: each aimed at one target from outside the ring,
    // spread by height so no two start together.
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    for (int32_t j = 0; j < shots; ++j)
    {
        int32_t t = j % targets;
        double a = 6.283185307179586 * (double)t / (double)targets;
        double dist = SceneRand(&rng, 5.0, 9.0);
        double sx = tx[t] + dist * cos(a) + SceneRand(&rng, -0.2, 0.2);
        double sz = tz[t] + dist * sin(a) + SceneRand(&rng, -0.2, 0.2);
        double sy = ty[t] + 0.9 * (double)(j / targets) + SceneRand(&rng, -0.2, 0.2);
        double speed = SceneRand(&rng, 25.0, 60.0);
        double dx = tx[t] - sx;
        double dy = ty[t] - sy;
        double dz = tz[t] - sz;
        double len = sqrt(dx * dx + dy * dy + dz * dz);
        bd.position = (m3Pos3){sx, sy, sz};
        bd.linearVelocity =
            (m3Vec3){(float)(speed * dx / len), (float)(speed * dy / len), (float)(speed * dz / len)};
        m3BodyId body = m3CreateBody(world, &bd);
        int32_t kind = j % 3;
        if (kind == 0)
        {
            m3Sphere ball = {{0.0f, 0.0f, 0.0f}, (float)SceneRand(&rng, 0.15, 0.35)};
            m3CreateSphereShape(body, &sd, &ball);
        }
        else if (kind == 1)
        {
            float h = (float)SceneRand(&rng, 0.15, 0.3);
            m3CreateBoxShape(body, &sd, (m3Vec3){h, h, h});
        }
        else
        {
            float hh = (float)SceneRand(&rng, 0.15, 0.3);
            m3Capsule cap = {{-hh, 0.0f, 0.0f}, {hh, 0.0f, 0.0f}, (float)SceneRand(&rng, 0.1, 0.2)};
            m3CreateCapsuleShape(body, &sd, &cap);
        }
    }
    return world;
}

// A plank (half extents 4.5 x 0.25 x 4.5) on the ground with `boxes`
// small boxes (half extent 0.35) on a grid on top of it, jittered by the
// seed, and a few spheres on top of the first boxes.  Every box touches
// the plank, so the plank's constraints outnumber the 16 graph colours.
static m3WorldId Plank(uint64_t seed, int32_t boxes)
{
    if (boxes < 17)
    {
        boxes = 17;
    }
    const int32_t spheres = 4;
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = boxes + spheres + 4;
    def.shapeCapacity = boxes + spheres + 4;
    m3WorldId world = m3CreateWorld(&def);
    SceneGround(world, 0.6f);
    uint64_t rng = seed ^ 0x9A4Cull;
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = 0.6f;
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    bd.position = (m3Pos3){0.0, 0.25, 0.0};
    m3BodyId plank = m3CreateBody(world, &bd);
    m3ShapeDef heavy = sd;
    heavy.density = 4.0f;
    m3CreateBoxShape(plank, &heavy, (m3Vec3){4.5f, 0.25f, 4.5f});
    int32_t side = 1;
    while (side * side < boxes)
    {
        side += 1;
    }
    const double pitch = 8.0 / (double)side;
    for (int32_t b = 0; b < boxes; ++b)
    {
        double x = -4.0 + pitch * (0.5 + (double)(b % side)) + SceneRand(&rng, -0.05, 0.05);
        double z = -4.0 + pitch * (0.5 + (double)(b / side)) + SceneRand(&rng, -0.05, 0.05);
        bd.position = (m3Pos3){x, 0.5 + 0.35 + SceneRand(&rng, 0.0, 0.02), z};
        m3BodyId body = m3CreateBody(world, &bd);
        m3CreateBoxShape(body, &sd, (m3Vec3){0.35f, 0.35f, 0.35f});
    }
    for (int32_t k = 0; k < spheres; ++k)
    {
        double x = -4.0 + pitch * (0.5 + (double)(k % side));
        double z = -4.0 + pitch * 0.5;
        bd.position = (m3Pos3){x, 1.2 + 0.3 + SceneRand(&rng, 0.0, 0.5), z};
        m3BodyId body = m3CreateBody(world, &bd);
        m3Sphere ball = {{0.0f, 0.0f, 0.0f}, 0.3f};
        m3CreateSphereShape(body, &sd, &ball);
    }
    return world;
}

// `count` spheres (radius U[0.3, 0.6]) and boxes (half extent U[0.3,
// 0.5]) with restitution U[0.3, 0.8] on a 1.6 m grid, dropped from 2-8 m
// onto a ground of restitution 0.5; every fourth body starts right above
// its neighbour so the two bounce off each other.
static m3WorldId Bounce(uint64_t seed, int32_t count)
{
    if (count < 2)
    {
        count = 2;
    }
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = count + 4;
    def.shapeCapacity = count + 4;
    m3WorldId world = m3CreateWorld(&def);
    m3BodyDef gd = m3DefaultBodyDef();
    m3BodyId ground = m3CreateBody(world, &gd);
    m3ShapeDef floorDef = m3DefaultShapeDef();
    floorDef.friction = 0.5f;
    floorDef.restitution = 0.5f;
    m3Plane floor = {{0.0f, 1.0f, 0.0f}, 0.0f};
    m3CreatePlaneShape(ground, &floorDef, &floor);
    uint64_t rng = seed ^ 0xB0B0ull;
    int32_t side = 1;
    while (side * side < count)
    {
        side += 1;
    }
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    for (int32_t k = 0; k < count; ++k)
    {
        m3ShapeDef sd = m3DefaultShapeDef();
        sd.friction = (float)SceneRand(&rng, 0.2, 0.8);
        sd.restitution = (float)SceneRand(&rng, 0.3, 0.8);
        double x = 1.6 * (double)(k % side);
        double z = 1.6 * (double)(k / side);
        double y = SceneRand(&rng, 2.0, 8.0);
        if (k % 4 == 3)
        {
            // Above the previous body, a little off its axis.
            x = 1.6 * (double)((k - 1) % side) + 0.15;
            z = 1.6 * (double)((k - 1) / side) - 0.1;
            y = 9.5 + SceneRand(&rng, 0.0, 1.5);
        }
        bd.position = (m3Pos3){x, y, z};
        bd.angularVelocity = (m3Vec3){(float)SceneRand(&rng, -1.0, 1.0), 0.0f,
                                      (float)SceneRand(&rng, -1.0, 1.0)};
        m3BodyId body = m3CreateBody(world, &bd);
        if (k % 2 == 0)
        {
            m3Sphere ball = {{0.0f, 0.0f, 0.0f}, (float)SceneRand(&rng, 0.3, 0.6)};
            m3CreateSphereShape(body, &sd, &ball);
        }
        else
        {
            float h = (float)SceneRand(&rng, 0.3, 0.5);
            m3CreateBoxShape(body, &sd, (m3Vec3){h, h, h});
        }
    }
    return world;
}

// Towers of 10 x 10 x 2 welded unit boxes on a grid of 16 m cells (the
// grid as square as the count allows), each box joined to its +x, +y
// and +z neighbours by a fixed joint with a 500 N force threshold, and
// four dense spheres per tower, each starting 12 m in front of a seeded
// target tower (+z side), 1-9 m up, flying at it at 20-40 m/s.
static m3WorldId City(uint64_t seed, int32_t towers)
{
    if (towers < 1)
    {
        towers = 1;
    }
    const int32_t nx = 10;
    const int32_t ny = 10;
    const int32_t nz = 2;
    const int32_t boxes = nx * ny * nz;
    const int32_t joints = (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1);
    const int32_t shots = 4 * towers;
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = boxes * towers + shots + 4;
    def.shapeCapacity = boxes * towers + shots + 4;
    def.jointCapacity = joints * towers + 4;
    m3WorldId world = m3CreateWorld(&def);
    SceneGround(world, 0.6f);
    uint64_t rng = seed ^ 0xC17Cull;
    int32_t side = 1;
    while (side * side < towers)
    {
        side += 1;
    }
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    m3ShapeDef sd = m3DefaultShapeDef();
    sd.friction = 0.6f;
    // One tower's bodies, indexed [y][z][x], reused per tower.
    static m3BodyId box[10][2][10];
    for (int32_t t = 0; t < towers; ++t)
    {
        const double cx = 16.0 * (double)(t % side);
        const double cz = 16.0 * (double)(t / side);
        for (int32_t y = 0; y < ny; ++y)
        {
            for (int32_t z = 0; z < nz; ++z)
            {
                for (int32_t x = 0; x < nx; ++x)
                {
                    bd.position = (m3Pos3){cx + (double)x - 4.5, 0.5 + (double)y,
                                           cz + (double)z - 0.5};
                    box[y][z][x] = m3CreateBody(world, &bd);
                    m3CreateBoxShape(box[y][z][x], &sd, (m3Vec3){0.5f, 0.5f, 0.5f});
                }
            }
        }
        for (int32_t y = 0; y < ny; ++y)
        {
            for (int32_t z = 0; z < nz; ++z)
            {
                for (int32_t x = 0; x < nx; ++x)
                {
                    for (int32_t axis = 0; axis < 3; ++axis)
                    {
                        const int32_t x2 = x + (axis == 0 ? 1 : 0);
                        const int32_t y2 = y + (axis == 1 ? 1 : 0);
                        const int32_t z2 = z + (axis == 2 ? 1 : 0);
                        if (x2 >= nx || y2 >= ny || z2 >= nz)
                        {
                            continue;
                        }
                        const m3Vec3 half = {axis == 0 ? 0.5f : 0.0f, axis == 1 ? 0.5f : 0.0f,
                                             axis == 2 ? 0.5f : 0.0f};
                        m3JointDef jd = m3DefaultJointDef();
                        jd.type = m3_fixedJoint;
                        jd.bodyA = box[y][z][x];
                        jd.bodyB = box[y2][z2][x2];
                        jd.localAnchorA = half;
                        jd.localAnchorB = (m3Vec3){-half.x, -half.y, -half.z};
                        m3JointId joint = m3CreateJoint(&jd);
                        m3Joint_SetBreakThresholds(joint, 500.0f, 0.0f);
                    }
                }
            }
        }
    }
    m3ShapeDef heavy = sd;
    heavy.density = 20.0f;
    for (int32_t k = 0; k < shots; ++k)
    {
        const int32_t target = (int32_t)(SceneSplitMix(&rng) % (uint64_t)towers);
        const double tx = 16.0 * (double)(target % side) + SceneRand(&rng, -4.0, 4.0);
        const double tz = 16.0 * (double)(target / side);
        const double y = SceneRand(&rng, 1.0, 9.0);
        const double speed = SceneRand(&rng, 20.0, 40.0);
        // Start 12 m out on the +z side, a little off line, aimed at the
        // tower's face.
        bd.position = (m3Pos3){tx + SceneRand(&rng, -1.0, 1.0), y, tz + 12.0 + 0.25 * (double)(k % 4)};
        bd.linearVelocity = (m3Vec3){0.0f, (float)SceneRand(&rng, 0.0, 2.0), (float)(-speed)};
        m3BodyId ball = m3CreateBody(world, &bd);
        m3Sphere shape = {{0.0f, 0.0f, 0.0f}, 0.5f};
        m3CreateSphereShape(ball, &heavy, &shape);
    }
    bd.linearVelocity = (m3Vec3){0.0f, 0.0f, 0.0f};
    return world;
}

// Height of the rain field's terrain at sample (x, z): four octaves of
// sin x cos, frequency doubling and weight halving per octave, scaled to
// a 4 m amplitude.
static double RainHeight(const double* ph, double x, double z)
{
    double h = 0.0;
    double weight = 1.0;
    double total = 0.0;
    double f = 0.045;
    for (int32_t o = 0; o < 4; ++o)
    {
        h += weight * sin(f * x + ph[2 * o]) * cos(f * z + ph[2 * o + 1]);
        total += weight;
        weight *= 0.5;
        f *= 2.0;
    }
    return 4.0 * h / total;
}

static m3WorldId Rain(uint64_t seed, int32_t bodies)
{
    if (bodies < 1)
    {
        bodies = 1;
    }
    const int32_t n = 255;
    const float cell = 1.0f;
    const double half = 0.5 * (double)(n - 1) * (double)cell;
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = bodies + 4;
    def.shapeCapacity = bodies + 4;
    def.jointCapacity = 4;
    m3WorldId world = m3CreateWorld(&def);
    uint64_t rng = seed ^ 0x4A1Full;
    double ph[8];
    for (int32_t k = 0; k < 8; ++k)
    {
        ph[k] = SceneRand(&rng, 0.0, 6.283185307179586);
    }
    static float heights[255 * 255];
    for (int32_t iz = 0; iz < n; ++iz)
    {
        for (int32_t ix = 0; ix < n; ++ix)
        {
            heights[iz * n + ix] = (float)RainHeight(ph, (double)ix, (double)iz);
        }
    }
    m3BodyDef gd = m3DefaultBodyDef();
    gd.position = (m3Pos3){-half, 0.0, -half};
    m3BodyId ground = m3CreateBody(world, &gd);
    m3ShapeDef hd = m3DefaultShapeDef();
    hd.friction = 0.6f;
    m3CreateHeightFieldGridShape(ground, &hd, heights, n, n, cell);
    int32_t side = 1;
    while (side * side < bodies)
    {
        side += 1;
    }
    const double spacing = 2.4;
    const double span = spacing * (double)(side - 1);
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    for (int32_t b = 0; b < bodies; ++b)
    {
        const double x = -0.5 * span + spacing * (double)(b % side) + SceneRand(&rng, -0.3, 0.3);
        const double z = -0.5 * span + spacing * (double)(b / side) + SceneRand(&rng, -0.3, 0.3);
        bd.position = (m3Pos3){x, SceneRand(&rng, 5.0, 100.0), z};
        m3BodyId body = m3CreateBody(world, &bd);
        m3ShapeDef sd = m3DefaultShapeDef();
        sd.density = (float)SceneRand(&rng, 0.5, 2.0);
        sd.friction = (float)SceneRand(&rng, 0.3, 0.9);
        const int32_t kind = b % 10;
        if (kind < 4)
        {
            m3Sphere ball = {{0.0f, 0.0f, 0.0f}, (float)SceneRand(&rng, 0.25, 0.75)};
            m3CreateSphereShape(body, &sd, &ball);
        }
        else if (kind < 7)
        {
            const float r = (float)SceneRand(&rng, 0.2, 0.5);
            const float hh = (float)SceneRand(&rng, 0.3, 1.0);
            m3Capsule cap = {{0.0f, -hh, 0.0f}, {0.0f, hh, 0.0f}, r};
            m3CreateCapsuleShape(body, &sd, &cap);
        }
        else
        {
            // 16-32 points uniform in the unit ball (rejection from the
            // cube), scaled by U[0.5, 1.5].
            m3Vec3 pts[32];
            const int32_t count = 16 + (int32_t)(SceneSplitMix(&rng) % 17u);
            const double scale = SceneRand(&rng, 0.5, 1.5);
            for (int32_t k = 0; k < count; ++k)
            {
                double px;
                double py;
                double pz;
                do
                {
                    px = SceneRand(&rng, -1.0, 1.0);
                    py = SceneRand(&rng, -1.0, 1.0);
                    pz = SceneRand(&rng, -1.0, 1.0);
                } while (px * px + py * py + pz * pz > 1.0);
                pts[k] = (m3Vec3){(float)(scale * px), (float)(scale * py), (float)(scale * pz)};
            }
            m3CreateHullShape(body, &sd, pts, count);
        }
    }
    return world;
}

static m3WorldId Mixed(uint64_t seed, int32_t bodies)
{
    if (bodies < 4)
    {
        bodies = 4;
    }
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = bodies + 4;
    def.shapeCapacity = bodies + 4;
    def.jointCapacity = 4;
    m3WorldId world = m3CreateWorld(&def);
    SceneGround(world, 0.6f);
    uint64_t rng = seed ^ 0x5E4Dull;
    const int32_t columns = (bodies + 3) / 4;
    int32_t side = 1;
    while (side * side < columns)
    {
        side += 1;
    }
    const double spacing = 1.6;
    const double span = spacing * (double)(side - 1);
    m3BodyDef bd = m3DefaultBodyDef();
    bd.type = m3_dynamicBody;
    for (int32_t b = 0; b < bodies; ++b)
    {
        const int32_t c = b / 4;
        const double x = -0.5 * span + spacing * (double)(c % side) + SceneRand(&rng, -0.1, 0.1);
        const double z = -0.5 * span + spacing * (double)(c / side) + SceneRand(&rng, -0.1, 0.1);
        const double y = 0.6 + 1.2 * (double)(b % 4) + SceneRand(&rng, 0.1, 0.4);
        bd.position = (m3Pos3){x, y, z};
        m3BodyId body = m3CreateBody(world, &bd);
        m3ShapeDef sd = m3DefaultShapeDef();
        sd.friction = (float)SceneRand(&rng, 0.4, 0.8);
        const int32_t kind = (int32_t)(SceneSplitMix(&rng) % 3u);
        if (kind == 0)
        {
            const float h = (float)SceneRand(&rng, 0.25, 0.5);
            m3CreateBoxShape(body, &sd, (m3Vec3){h, h, h});
        }
        else if (kind == 1)
        {
            m3Sphere ball = {{0.0f, 0.0f, 0.0f}, (float)SceneRand(&rng, 0.25, 0.5)};
            m3CreateSphereShape(body, &sd, &ball);
        }
        else
        {
            m3Vec3 pts[16];
            const double scale = SceneRand(&rng, 0.3, 0.6);
            for (int32_t k = 0; k < 16; ++k)
            {
                double px;
                double py;
                double pz;
                double rr;
                do
                {
                    px = SceneRand(&rng, -1.0, 1.0);
                    py = SceneRand(&rng, -1.0, 1.0);
                    pz = SceneRand(&rng, -1.0, 1.0);
                    rr = px * px + py * py + pz * pz;
                } while (rr > 1.0 || rr < 0.04);
                const double inv = scale / sqrt(rr);
                pts[k] = (m3Vec3){(float)(inv * px), (float)(inv * py), (float)(inv * pz)};
            }
            m3CreateHullShape(body, &sd, pts, 16);
        }
    }
    return world;
}

// Build one seeded scene; returns the null world id for an unknown
// scene number.
M3S_API m3WorldId m3s_build(int32_t scene, uint64_t seed, int32_t param)
{
    switch (scene)
    {
    case M3S_SPHERE_PYRAMID:
        return SphereLayers();
    case M3S_BOX_PYRAMID:
        return BoxWall(param > 0 ? param : 20);
    case M3S_UNEVEN:
        return UnevenWorld(seed, param);
    case M3S_FREEFALL:
        return FreeFall(param > 0 ? param : 8);
    case M3S_TOWERS:
        return Towers(seed, param > 0 ? param : 4);
    case M3S_TERRAIN:
        return Terrain(seed, param > 0 ? param : 60);
    case M3S_SHOTS:
        return Shots(seed, param > 0 ? param : 24);
    case M3S_PLANK:
        return Plank(seed, param > 0 ? param : 25);
    case M3S_BOUNCE:
        return Bounce(seed, param > 0 ? param : 40);
    case M3S_CITY:
        return City(seed, param > 0 ? param : 1000);
    case M3S_RAIN:
        return Rain(seed, param > 0 ? param : 10000);
    case M3S_MIXED:
        return Mixed(seed, param > 0 ? param : 1000);
    default:
    {
        m3WorldId none = {0, 0};
        return none;
    }
    }
}

// Body count the uneven-world generator produces for world `index` of
// a batch seeded by `seed`: log-uniform in [lo, hi].
M3S_API int32_t m3s_uneven_size(uint64_t seed, int32_t index, int32_t lo, int32_t hi)
{
    uint64_t s = seed ^ (0xA0761D6478BD642Full * (uint64_t)(index + 1));
    double u = SceneRand(&s, 0.0, 1.0);
    double n = exp(log((double)lo) + u * (log((double)hi) - log((double)lo)));
    int32_t b = (int32_t)n;
    return b < lo ? lo : (b > hi ? hi : b);
}
