"""The backend's host-side SpatiallyExplicit tables are bit-identical to the
oracle's restatement of InMemoryPackedSeparableAliasDispersalSampler::new
(CPU, no GPU needed)."""
import numpy as np
import pytest


def compare(nb, oracle, syn, desc):
    ref = oracle.build_alias(desc)
    cells, atoms = nb.build_tables(syn.to_scenario(desc))
    assert np.array_equal(cells["atom_start"].astype(np.uint64), ref["range_start"])
    assert np.array_equal((cells["atom_start"] + cells["atom_count"]).astype(np.uint64),
                          ref["range_end"])
    assert np.array_equal(cells["self_dispersal"].view(np.uint64),
                          ref["self_dispersal"].view(np.uint64))
    assert np.array_equal(cells["non_self_event"].astype(np.uint64), ref["non_self_event"])
    assert np.array_equal(atoms["u"].view(np.uint64), ref["atom_u"].view(np.uint64))
    assert np.array_equal(atoms["e"], ref["atom_e"])
    assert np.array_equal(atoms["k"], ref["atom_k"])
    hab = np.asarray(desc["habitat"], dtype=np.uint64).reshape(-1)
    assert np.array_equal(cells["habitat"], hab)
    assert np.array_equal(cells["injection"], np.concatenate([[0], np.cumsum(hab)[:-1]]))
    return cells, atoms


@pytest.mark.parametrize("w,h,sigma,seed", [(6, 5, 1.0, 1), (8, 8, 1.5, 2), (16, 16, 3.0, 3),
                                            (32, 32, 3.0, 4)])
def test_tables_match_oracle(nb, oracle, syn, w, h, sigma, seed):
    hab = syn.habitat_map(w, h, 0.15, 30, seed)
    compare(nb, oracle, syn, dict(kind=3, speciation_probability=1e-3, width=w, height=h,
                                  habitat=hab, dispersal=syn.dispersal_map(hab, sigma)))


def test_self_dispersal_edge_rows(nb, oracle, syn):
    """Rows with only self-dispersal (sd == 1), with dominant self-dispersal
    (removed from the atoms, sd_u >= 1) and with none (non-habitat)."""
    hab = np.array([[3, 0, 2], [1, 4, 5]], dtype=np.uint32)
    n = hab.size
    d = np.zeros((n, n))
    d[0, 0] = 1.0                        # self only
    d[2, [2, 3, 4]] = [0.9, 0.05, 0.05]  # dominant self
    d[3, [0, 4, 5]] = [0.2, 0.3, 0.5]    # no self
    d[4, [4, 5]] = [0.1, 0.9]            # small self, stays in the atoms
    d[5, [0, 2, 3, 4, 5]] = 0.2
    desc = dict(kind=3, speciation_probability=1e-3, width=3, height=2, habitat=hab, dispersal=d)
    cells, atoms = compare(nb, oracle, syn, desc)
    assert cells["self_dispersal"][0] == 1.0 and cells["atom_count"][0] == 0
    assert cells["non_self_event"][2] == 2        # self-dispersal kept out of the atoms
    assert cells["atom_count"][1] == 0            # non-habitat row


def test_contract_violations(nb, syn):
    hab = np.array([[1, 0], [1, 1]], dtype=np.uint32)
    d = np.full((4, 4), 0.25)
    with pytest.raises(nb.NecsimError) as e:        # dispersal into and from non-habitat
        nb.build_tables(nb.SpatiallyExplicit(hab, d))
    assert e.value.code == -6
    with pytest.raises(nb.NecsimError) as e:
        nb.build_tables(nb.SpatiallyExplicit(np.zeros((2, 2), np.uint32), np.zeros((4, 4))))
    assert e.value.code == -7
