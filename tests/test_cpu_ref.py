"""The oracle's C++ CPU arm (the timed CPU baseline) against the NumPy oracle:
the per-unit RI-MP2 energy + adjoint, DF-J and DF-K on small seeded inputs.
Also that the units partition the pair loop (any unit width gives the same
energy) and the physical-core count is positive."""
import numpy as np

from oracle import cpu_ref, dfjk, rimp2, synthetic


def test_rimp2_units_match_oracle():
    b, eo, ev = synthetic.rimp2_inputs(150, 7, 31)
    e_os, e_ss, gamma, d_o, d_v = rimp2.energy_gamma_deps(b, eo, ev)
    for width in (1, 3, 7):
        c_os, c_ss, c_g, c_do = cpu_ref.rimp2_energy_grad(b, eo, ev, width=width)
        assert abs(c_os - e_os) <= 1e-12 * abs(e_os) and abs(c_ss - e_ss) <= 1e-12 * abs(e_os)
        assert np.abs(c_g - gamma).max() <= 1e-12 * np.abs(gamma).max()
        assert np.abs(c_do - d_o).max() <= 1e-12 * np.abs(d_o).max()


def test_rimp2_units_threads_independent():
    b, eo, ev = synthetic.rimp2_inputs(120, 6, 25)
    units = [(i, j0, min(6, j0 + 2)) for i in range(6) for j0 in range(0, 6, 2)]
    _, e1, _ = cpu_ref.rimp2_units(b, eo, ev, units, 1)
    _, e4, _ = cpu_ref.rimp2_units(b, eo, ev, units, 4)
    assert np.array_equal(e1, e4)


def test_dfjk_match_oracle():
    b, c, d = synthetic.dfjk_inputs(40, 90, 6)
    bp = dfjk.pack_lower(b)
    _, jp = cpu_ref.dfj(bp, dfjk.packed_density_weights(d), 3)
    j = dfjk.unpack_symmetric(jp, 40)
    j_ref = dfjk.df_j_square(b, d)
    assert np.abs(j - j_ref).max() <= 1e-12 * np.abs(j_ref).max()
    _, k = cpu_ref.dfk(b, c, 3, qchunk=7)
    k_ref = dfjk.df_k_occ(b, c)
    assert np.abs(k - k_ref).max() <= 1e-12 * np.abs(k_ref).max()
    assert np.array_equal(k, k.T)


def test_physical_cores():
    assert cpu_ref.physical_cores() >= 1
