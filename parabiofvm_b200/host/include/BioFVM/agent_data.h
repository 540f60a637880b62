// Agent data in structure-of-arrays form (include/BioFVM/agent_data.h of the reference): per-agent
// rows of `substrates_count` values, volumes and `dims` coordinates.  These are the arrays the
// solver copies to the GPU as they are.
#pragma once

#include <vector>

#include "types.h"

namespace biofvm {

struct microenvironment;

struct agent_data
{
	std::vector<real_t> secretion_rates;
	std::vector<real_t> saturation_densities;
	std::vector<real_t> uptake_rates;
	std::vector<real_t> net_export_rates;

	std::vector<real_t> internalized_substrates;
	std::vector<real_t> fraction_released_at_death;
	std::vector<real_t> fraction_transferred_when_ingested;

	std::vector<real_t> volumes;
	std::vector<real_t> positions;

	index_t agents_count;

	microenvironment& m;

	explicit agent_data(microenvironment& m);

	// append one agent (zeroed rows)
	void add();
	// remove agent `index`; the last agent takes its place
	void remove(index_t index);
};

} // namespace biofvm
