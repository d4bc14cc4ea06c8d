/* Declarations only (see spmacc/particles/algorithms/InteractParticles.hpp here). */
#pragma once
#include <spmacc/particles/algorithms/InteractParticles.hpp>
