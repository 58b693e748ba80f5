"""The benchmark workload is the one bench.py describes: the atom + rigid
rotor system, JTOT = 0..80 in both parity blocks (161 non-empty blocks,
N = 5..36), 4000 MDPROP steps from 2.5 to 40 Angstrom, seeded energies in
1-500 cm-1, every job an (energy, block) pair with its WKB initial Y."""
import numpy as np

from molscat_b200 import systems as S


def test_batched_workload_shape():
    wl = S.batched_workload(n_energies=2)
    ns = np.array([c.n for c in wl.systems])
    assert len(wl.systems) == 161
    assert ns.min() == 5 and ns.max() == 36
    assert wl.njobs == 2 * 161
    sysm = S.rotor_system()
    for g in wl.segments:
        assert g.nstep == S.ROTOR_NSTEP == 4000
        assert abs(g.rtab[0] * sysm.rm - 2.5) < 1e-12
        assert abs(g.rtab[-1] * sysm.rm - 40.0) < 1e-9
    # jobs of a block are consecutive and every job has a symmetric N x N start
    assert np.all(np.diff(wl.job_sys) >= 0)
    for j in (0, wl.njobs - 1):
        y0 = wl.job_y0[j]
        n = wl.systems[wl.job_sys[j]].n
        assert y0.shape == (n, n) and np.array_equal(y0, y0.T)
    # the work metric: sum over jobs of N^3 * NSTEP
    assert wl.channel3_steps() == float(sum(int(ns[s]) ** 3 * 4000 for s in wl.job_sys))


def test_batched_energies_are_seeded_in_range():
    e = S.batched_energies(512)
    assert e.shape == (512,) and e.min() >= 1.0 and e.max() <= 500.0
    assert np.array_equal(e, S.batched_energies(512))
    assert not np.array_equal(e, S.batched_energies(512, seed=1))
