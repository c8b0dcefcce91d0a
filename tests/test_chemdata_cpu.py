"""Mechanism tables on the CPU: the reference's non-reacting 4-species set
(H2_mech_mixing.inp, parsed into data/h2_mixing_4sp.json) is exactly the
H2-air mechanism's species data re-indexed, and the derived mechanisms of
other species counts (subsets, inert copies) are well formed."""
import numpy as np

import chemdata


def test_mixing_set_is_the_reindexed_species_data():
    m9 = chemdata.h2_air_9sp()
    m4 = chemdata.h2_mixing_4sp()
    assert m4.names == ["H2", "H2O", "O2", "N2"] and m4.n_reac == 0
    s4 = chemdata.subset(m9, m4.names, reactions=False)
    for k, v in m4.tables.items():
        assert np.array_equal(v, s4.tables[k]), k


def test_reacting_subset_keeps_the_reactions_among_its_species():
    m9 = chemdata.h2_air_9sp()
    keep = ["H2", "H", "O2", "O", "OH", "H2O", "N2"]
    m7 = chemdata.subset(m9, keep)
    assert m7.n_spec == 7 and m7.n_reac == 8
    drop = [m9.names.index(n) for n in ("HO2", "H2O2")]
    kept = [r for r in range(m9.n_reac) if not any(m9.tables["stoi_f"][r, d] or m9.tables["stoi_b"][r, d]
                                                   for d in drop)]
    ix = [m9.names.index(n) for n in keep]
    assert np.array_equal(m7.tables["stoi_f"], m9.tables["stoi_f"][kept][:, ix])
    assert np.array_equal(m7.tables["A"], m9.tables["A"][kept])


def test_inert_copies_reach_every_species_count():
    m9 = chemdata.h2_air_9sp()
    for k in (1, 3, 11):
        m = chemdata.with_inert_copies(m9, "N2", k)
        ns = 9 + k
        assert m.n_spec == ns and m.n_reac == m9.n_reac
        assert m.tables["binary_diffusivity_coeff"].shape == (ns, ns)
        assert m.tables["stoi_f"].shape == (m9.n_reac, ns) and not m.tables["stoi_f"][:, 9:].any()
        n2 = m9.names.index("N2")
        assert np.array_equal(m.tables["third_body_coeff"][:, 9:],
                              np.repeat(m9.tables["third_body_coeff"][:, n2:n2 + 1], k, axis=1))
