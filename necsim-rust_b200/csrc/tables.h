// tables.h -- host construction of the SpatiallyExplicit device tables.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/necsim_b200.h"
#include "layout.h"

namespace necsim {

struct HostTables {
    std::vector<CellRecord> cells;  // one per habitat-map cell
    std::vector<AliasAtom> atoms;   // packed per cell, in the reference's atom order
    // Shannon entropy (nats) of each cell's dispersal distribution
    // p(c) = w(c) / sum(w), w(c) = dispersal(r, c) * habitat(c): a feature of
    // the learned lifetime model (0 for non-habitat cells)
    std::vector<float> entropy;
};

// Builds the packed separable alias tables of a SpatiallyExplicit scenario
// (InMemoryPackedSeparableAliasDispersalSampler::new,
// necsim/impls/no-std/src/cogs/dispersal_sampler/in_memory/packed_separable_alias/mod.rs:64-203)
// and the habitat injection prefix (habitat/in_memory.rs:143-163), rows in
// parallel on `threads` host threads (0: all cores).
// Returns 0, or 1 empty habitat, 2 dispersal contract violated, 3 too many atoms.
int build_spatially_explicit_tables(const necsim_scenario &sc, HostTables &out, unsigned threads = 0);

// The Shannon entropy (nats) of cell r's dispersal distribution, as the
// table build records it (0 without a dispersal map or from a non-habitat cell).
float dispersal_entropy(const necsim_scenario &sc, uint64_t r);

// check_in_memory_dispersal_contract (dispersal_sampler/in_memory/contract.rs:13-69).
bool dispersal_contract_holds(const necsim_scenario &sc);

}  // namespace necsim
