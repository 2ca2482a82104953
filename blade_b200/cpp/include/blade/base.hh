// Umbrella header of the C++ host layer: types, memory, modules, bundles, Pipeline, Runner.
// Link with libblade_b200.so (built by `python -m blade_b200.build`).
#ifndef BLADE_B200_BASE_HH
#define BLADE_B200_BASE_HH

#include "blade/types.hh"
#include "blade/memory.hh"
#include "blade/module.hh"
#include "blade/modules.hh"
#include "blade/bundles.hh"
#include "blade/pipeline.hh"

#endif
