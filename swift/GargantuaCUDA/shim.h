/* Umbrella header of the GargantuaCUDA module.
 *
 * Inside gargantua's own package, define GG_WITH_HOST_SHADER_TYPES (e.g.
 * cSettings: [.define("GG_WITH_HOST_SHADER_TYPES")]) and put the
 * ShaderTypes target's include directory on the search path: the host's
 * ShaderTypes.h is then included first and gargantua_types.h keeps its
 * structs (Particle, SimUniforms, SplatUniforms, MarchUniforms, RayProbe,
 * ...), so a Swift file that imports both ShaderTypes and GargantuaCUDA
 * passes its own values to gg_* unchanged. Standalone, the library's own
 * definitions of the same layouts are used. */
#ifndef GARGANTUA_CUDA_SHIM_H
#define GARGANTUA_CUDA_SHIM_H
#ifdef GG_WITH_HOST_SHADER_TYPES
#include <ShaderTypes.h>
#endif
#include "../../include/gargantua.h"
#endif
