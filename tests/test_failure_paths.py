"""Failure paths of the boundary, made on the host so that no GPU faults.

The reference maps its CUDA failures to error values
(rustcoalescence/algorithms/cuda/src/error.rs:1-93); this backend returns
NECSIM_E_* codes and never aborts across the C ABI:
  * the round watchdog (necsim_args.max_rounds) ends a run that needs more
    rounds with NECSIM_E_TIMEOUT;
  * SpatiallyExplicit tables handed over by the caller are not range-checked
    on the host: the kernels bound-check every cell and atom index before
    reading it, and a planted out-of-range index ends the run with
    NECSIM_E_DEVICE_CHECK (nothing is read out of range: the check comes
    before the load).
"""
import numpy as np
import pytest

from test_gpu_parity import same_stream

E_DEVICE_CHECK = -4
E_TIMEOUT = -5
E_INVALID_ARGUMENT = -1


def se_landscape(syn, w=12, h=10, seed=3):
    hab = syn.habitat_map(w, h, 0.15, 20, seed)
    return hab, syn.dispersal_map(hab, 2.0)


def test_tables_argument_mirrors_header(nb):
    """The ctypes mirror carries the new trailing fields in the header's order."""
    names = [f for f, _ in nb.CScenario._fields_]
    assert names[-3:] == ["cells", "atoms", "n_atoms"]
    assert [f for f, _ in nb.CArgs._fields_][-6:] == ["max_rounds", "priority_sims", "priority_groups",
                                                      "priority_list", "reserve_sms", "priority_engines"]
    assert nb.lib().necsim_abi_version() == 3
    assert nb._args_struct(nb.CUDA(reserve_sms=8)).reserve_sms == 8
    assert nb._args_struct(nb.CUDA()).reserve_sms == 0
    assert nb._args_struct(nb.CUDA(priority_engines=2)).priority_engines == 2


def test_scenario_needs_a_dispersal_map_or_tables(nb, syn):
    hab, _ = se_landscape(syn)
    with pytest.raises(ValueError):
        nb.simulate(1e-3, nb.SpatiallyExplicit(hab, None), 1)


@pytest.mark.gpu
def test_round_watchdog_times_out(nb, syn):
    desc, seed = syn.config1()
    with pytest.raises(nb.NecsimError) as e:
        # checked between graph launches: two rounds per graph, so at most 4 rounds run
        nb.simulate(desc["speciation_probability"], syn.to_scenario(desc), seed,
                    nb.CUDA(max_rounds=4, rounds_per_graph=2))
    assert e.value.code == E_TIMEOUT
    # the same run within its round count completes
    ok = nb.simulate(desc["speciation_probability"], syn.to_scenario(desc), seed)
    again = nb.simulate(desc["speciation_probability"], syn.to_scenario(desc), seed,
                        nb.CUDA(max_rounds=ok.n_rounds + 64))
    assert (again.steps, again.biodiversity) == (ok.steps, ok.biodiversity)


@pytest.mark.gpu
def test_prebuilt_tables_equal_map_built_tables(nb, syn):
    hab, disp = se_landscape(syn)
    cells, atoms = nb.build_tables(nb.SpatiallyExplicit(hab, disp))
    a = nb.simulate(2e-3, nb.SpatiallyExplicit(hab, disp), 5)
    b = nb.simulate(2e-3, nb.SpatiallyExplicit(hab, None, tables=(cells, atoms)), 5)
    assert same_stream(a.speciation, b.speciation)
    assert (a.steps, a.biodiversity, a.n_dedup, a.time) == (b.steps, b.biodiversity, b.n_dedup, b.time)


@pytest.mark.gpu
def test_atom_range_outside_the_table_is_a_device_check(nb, syn):
    hab, disp = se_landscape(syn)
    cells, atoms = nb.build_tables(nb.SpatiallyExplicit(hab, disp))
    bad = cells.copy()
    live = bad["atom_count"] > 0
    assert live.any()
    bad["atom_start"][live] = len(atoms)  # every alias draw indexes past the table
    bad["self_dispersal"][live] = 0.0     # and every dispersal uses the alias
    with pytest.raises(nb.NecsimError) as e:
        nb.simulate(2e-3, nb.SpatiallyExplicit(hab, None, tables=(bad, atoms)), 5)
    assert e.value.code == E_DEVICE_CHECK


@pytest.mark.gpu
def test_atom_target_outside_the_map_is_a_device_check(nb, syn):
    hab, disp = se_landscape(syn)
    cells, atoms = nb.build_tables(nb.SpatiallyExplicit(hab, disp))
    cells = cells.copy()
    live = cells["atom_count"] > 0
    cells["self_dispersal"][live] = 0.0
    bad = atoms.copy()
    bad["e"] = 0xFFFFFFF0  # no such cell
    bad["k"] = 0xFFFFFFF0
    with pytest.raises(nb.NecsimError) as e:
        nb.simulate(2e-3, nb.SpatiallyExplicit(hab, None, tables=(cells, bad)), 5)
    assert e.value.code == E_DEVICE_CHECK


def test_outcome_conversion_keeps_every_field(nb):
    """The ctypes outcome converts field by field: events and lineages stay
    in their own attributes beside the timeline fields."""
    o = nb.COutcome()
    o.paused, o.time, o.steps, o.n_initial, o.n_remaining = 1, 2.5, 7, 9, 3
    o.resident_ms, o.end_ms, o.routed_ms = 1.5, 4.25, -1.0
    spec = np.zeros(2, dtype=nb.SPECIATION_DTYPE)
    rem = np.zeros(3)
    out = nb._outcome(o, spec, rem)
    assert out.speciation is spec and out.remaining is rem
    assert (out.paused, out.time, out.steps, out.n_initial, out.n_remaining) == (True, 2.5, 7, 9, 3)
    assert (out.resident_ms, out.end_ms, out.routed_ms) == (1.5, 4.25, -1.0)
