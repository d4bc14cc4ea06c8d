/* Host-only stand-in for the reference's alpaka function specifiers.
 * Lets the reference's header-only physics (SPH kernels, EOS, pair functors)
 * compile with plain g++ for the CPU oracle; it carries no reference code. */
#pragma once
#define HDINLINE inline
#define DINLINE inline
#define HINLINE inline
#define DEVICEONLY
#define PMACC_CUDA_ARCH 0
