// Scene-generator API shim for the oracle build: the product's seeded
// scene generator (maul3d_b200/csrc/scenes.c) compiles against the
// reference engine's own public headers here, so the oracle and the
// device path build their worlds from the same source and seeds.
#ifndef M3_SCENE_API_H
#define M3_SCENE_API_H
#include "maul3d/world.h"
#include "maul3d/body.h"
#include "maul3d/shape.h"
#include "maul3d/joint.h"
#define M3S_API __attribute__((visibility("default")))
#endif
