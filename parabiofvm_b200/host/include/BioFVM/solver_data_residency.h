// Where a microenvironment's data currently lives (include/BioFVM/solver_data_residency.h of the
// reference): the member microenvironment::data_residency, host on construction.
#pragma once

namespace biofvm {
namespace solvers {

enum class data_residency
{
	host,
	device
};

} // namespace solvers
} // namespace biofvm
