"""Host-side input formats of the reference, mirrored in lpm-cpp_b200/lpm.py: the LAMMPS-style
dump read by Assembly::readDump (include/assembly.h:338-388) and the bond file read by
Assembly::readBond (include/assembly.h:391-424) and written by Assembly::writeBond (:269-283).
No GPU: these run before a solver exists."""
import os

import numpy as np
import pytest

from _util import CFG, LPM, O, oracle_problem


def _write_dump(path, xyz, types, box, fmt="%.4e"):
    # the layout of Assembly::writeConfigurationDump (include/assembly.h:285-307)
    with open(path, "w") as f:
        f.write("ITEM: TIMESTEP\n0\nITEM: NUMBER OF ATOMS\n%d\nITEM: BOX BOUNDS pp pp pp\n" % len(xyz))
        for k in range(3):
            f.write("%8.8f %8.8f\n" % (box[2 * k], box[2 * k + 1]))
        f.write("ITEM: ATOMS id type x y z\n")
        for i, (p, t) in enumerate(zip(xyz, types)):
            f.write(("%d %d " + " ".join([fmt] * 3) + " \n") % (i, t, *p))


def test_read_dump_parses_like_fscanf(tmp_path):
    case = CFG.hex_plate(size=1.0, radius=0.1, steps=1)
    types = np.arange(case.n, dtype=np.int32) % 3
    path = str(tmp_path / "plate.dump")
    _write_dump(path, case.xyz, types, case.box)
    cell = LPM.UnitCell(LPM.LatticeType.Hexagon2D, 0.1)
    a = LPM.Assembly.fromDump(path, cell, LPM.ParticleType.Elastic)
    expect = np.array([[float("%.4e" % v) for v in p] for p in case.xyz])
    assert np.array_equal(a.xyz, expect)
    assert np.array_equal(a.type, types)
    assert a.box == pytest.approx(case.box)
    assert a.bonds is None


def test_read_dump_rejects_ids_out_of_order(tmp_path):
    path = str(tmp_path / "bad.dump")
    _write_dump(path, np.zeros((2, 3)), [0, 0], [0, 1, 0, 1, 0, 1])
    txt = open(path).read().replace("\n0 0 ", "\n7 0 ")
    open(path, "w").write(txt)
    with pytest.raises(ValueError):
        LPM.Assembly.fromDump(path, LPM.UnitCell(LPM.LatticeType.Hexagon2D, 0.1))
    with pytest.raises(FileNotFoundError):
        LPM.Assembly.fromDump(str(tmp_path / "missing.dump"), LPM.UnitCell(LPM.LatticeType.Hexagon2D, 0.1))


def _shuffled_bond_file(path, bonds, seed):
    O.write_bond_file(path, *bonds)
    rows = np.loadtxt(path, dtype=np.int64, ndmin=2)
    rows = rows[np.random.default_rng(seed).permutation(len(rows))]
    np.savetxt(path, rows, fmt="%d")
    # expected lists: per particle, per layer, partners in the shuffled file order
    nb0, nb1, p2 = [], [], []
    n = len(bonds[0])
    for i in range(n):
        for L, cnt in ((0, nb0), (1, nb1)):
            sel = rows[(rows[:, 2] == i) & (rows[:, 1] == L), 3]
            cnt.append(len(sel))
            p2.extend(sel.tolist())
    return np.array(nb0, np.int32), np.array(nb1, np.int32), np.array(p2, np.int32)


def test_read_bond_keeps_file_order_and_round_trips(tmp_path):
    case = CFG.notched_plate(size=1.6, radius=0.1, crack=0.3, steps=1)
    path = str(tmp_path / "plate.bond")
    expect = _shuffled_bond_file(path, case.bonds, seed=5)
    a = case.assembly()
    a.readBond(path)
    for x, y in zip(a.bonds, expect):
        assert np.array_equal(x, y)
    out = str(tmp_path / "again.bond")
    a.writeBond(out)
    b = case.assembly()
    b.readBond(out)
    for x, y in zip(b.bonds, expect):
        assert np.array_equal(x, y)
    bad = str(tmp_path / "bad.bond")
    open(bad, "w").write("0 2 0 1\n")
    with pytest.raises(ValueError):
        case.assembly().readBond(bad)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/lpm_ref not built (make -C oracle ref)")
def test_reference_reads_shuffled_bond_file_like_the_mirror(tmp_path):
    """The reference's own readBond on a shuffled file builds the lists the mirror reads, and
    the oracle given those lists reproduces its topology, initial forces and stiffness."""
    case = CFG.notched_plate(size=1.6, radius=0.1, crack=0.3, steps=1, total_disp=0.0005)
    d = str(tmp_path / "ref")
    os.makedirs(d)
    bond_path = str(tmp_path / "shuffled.bond")
    expect = _shuffled_bond_file(bond_path, case.bonds, seed=11)
    spec = O.write_ref_spec(case, d, dump_k=(0,), cg_tol=(1e-24, 0.0), tol_iter=1e-9)
    spec = "\n".join(ln for ln in spec.splitlines() if not ln.startswith("bondfile")) + f"\nbondfile {bond_path}\n"
    O.run_ref(spec, d, threads=1)
    assert np.array_equal(O.read_bin(d, "nb0.i32", np.int32), expect[0])
    assert np.array_equal(O.read_bin(d, "nb1.i32", np.int32), expect[1])
    assert np.array_equal(O.read_bin(d, "bond_p2.i32", np.int32), expect[2])
    case.bonds = expect
    o = oracle_problem(case, cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    assert np.array_equal(o.conns()[2], O.read_bin(d, "conns.i32", np.int32))
    o.update_geometry()
    o.update_force_state()
    assert np.array_equal(o.state()["pin"].reshape(-1), O.read_bin(d, "pin_init.f64", np.float64))
    from _util import oracle_step_args
    ok, _ = o.solve_load_step(*oracle_step_args(case, 0))
    assert ok
    assert np.array_equal(o.export_csr()[3], O.read_bin(d, "K_000.f64", np.float64))
