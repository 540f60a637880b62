// agent_container_base and agent_container_common (include/BioFVM/agent_container_base.h of the
// reference) are declared with the concrete agent_container in agent_container.h.
#pragma once

#include "agent_container.h"
