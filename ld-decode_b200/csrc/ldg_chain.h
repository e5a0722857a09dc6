// Host field chain: types come from the public ABI header.
#pragma once
#include "ldgpu.h"

typedef ldg_chain_params LdgChainParams;
typedef ldg_chain_state LdgChainState;
typedef ldg_field_plan LdgFieldPlan;
