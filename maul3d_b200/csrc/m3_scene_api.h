// Scene-generator API for the product build: the seeded scenes in
// scenes.c use only the reference-named public API, declared for this
// library by include/maul3d_b200.h.
#ifndef M3_SCENE_API_H
#define M3_SCENE_API_H
#include "maul3d_b200.h"
#define M3S_API __attribute__((visibility("default")))
#endif
