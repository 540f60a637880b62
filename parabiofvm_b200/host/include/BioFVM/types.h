// Basic types of the paraBioFVM host API (include/BioFVM/types.h of the reference): 32-bit
// indices, FP32 reals and fixed-size points.  The GPU library computes in FP32 only, so the
// reference's USE_DOUBLES build option has no counterpart here.
#pragma once

#include <array>
#include <cstdint>

#ifdef USE_DOUBLES
	#error "the B200 microenvironment library computes in FP32; USE_DOUBLES is not supported"
#endif

namespace biofvm {

using agent_id_t = uint32_t;
using index_t = int32_t;
using real_t = float;

template <typename T, int dims>
using point_t = std::array<T, dims>;

} // namespace biofvm
