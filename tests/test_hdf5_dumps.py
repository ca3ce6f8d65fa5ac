"""HDF5 field dumps (mp_hdf5_*): MPulse's FieldDiag output through HDFostream.

CPU part: the file-name convention of DiagnosticInterface::parsedFileName
(diagnostic.cpp:52-70), and files of host arrays read back with the format
reader of tests/hdf5_subset.py (dataset names "data0", "data1", ... as
HDFstream::getNextBlockName gives them, sorted symbol table nodes across more
than one node, dims, values)."""
import os

import numpy as np
import pytest

from mpulse_b200 import abi, runtime
from tests.hdf5_subset import read_datasets

pytestmark = pytest.mark.skipif(not os.path.exists(runtime.LIB_PATH), reason="library not built")


@pytest.mark.parametrize("pattern,proc,time,want", [
    ("out.h5", 0, 5, "out.h5"),
    ("Ex#t.h5", 0, 120, "Ex120.h5"),
    ("f_#p_#t.h5", 3, 7, "f_3_7.h5"),
    ("f_#t_#t_#p#p.h5", 2, 9, "f_9_#t_2#p.h5"),  # only the first of each is replaced
])
def test_file_name_substitution(pattern, proc, time, want):
    assert runtime.diag_file_name(pattern, proc, time) == want


@pytest.mark.parametrize("count", [1, 3, 12, 40])
def test_host_arrays_round_trip(tmp_path, count):
    rng = np.random.default_rng(count)
    arrays = [rng.standard_normal((3 + q % 4, 5, 2 + q % 3)) for q in range(count)]
    name = runtime.write_hdf5_arrays(str(tmp_path / "dump_#t.h5"), arrays, time=count)
    assert name.endswith(f"dump_{count}.h5")
    got = read_datasets(name)
    want_names = [f"data{q}" for q in range(count)]
    assert sorted(got) == sorted(want_names)
    for q, a in enumerate(arrays):
        np.testing.assert_array_equal(got[want_names[q]], a)


def test_file_without_datasets(tmp_path):
    """An HDFostream that writes nothing (a slice on the boundary) leaves a
    file whose root group has no entries."""
    with runtime.Hdf5File(str(tmp_path / "empty.h5")) as f:
        pass
    assert read_datasets(f.name) == {}


def test_too_many_datasets_is_an_error(tmp_path):
    arrays = [np.zeros((1, 1, 1))] * 257
    with pytest.raises(runtime.MPulseError) as e:
        runtime.write_hdf5_arrays(str(tmp_path / "big.h5"), arrays)
    assert e.value.code == abi.MP_ERR_INVALID


def _reference_records(path):
    """The datasets MPulse's HDFostream handed to the HDF5 stand-in for the
    file `path`: {name: array [k][j][i]} (the stand-in's grid is C order over
    (i, j, k); the dataspace MPulse declares is the reversed {nz+2, ny+2,
    nx+2}; a slice likewise, rank 2)."""
    raw = open(path + ".raw", "rb").read()
    out = {}
    for line in open(path + ".calls"):
        parts = line.split()
        assert parts[0] == "dataset" and parts[2] == "3"  # H5T_NATIVE_DOUBLE
        rank = int(parts[3])
        dims = tuple(int(x) for x in parts[4:4 + rank])
        off, nbytes = int(parts[4 + rank]), int(parts[5 + rank])
        a = np.frombuffer(raw, dtype=np.float64, count=nbytes // 8, offset=off)
        out[parts[1]] = a.reshape(dims[::-1]).T
        assert out[parts[1]].shape == dims
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["nonlin_all_short", "plasma_nonlin_all_short"])
def test_dumps_match_mpulse_fielddiag(tmp_path, monkeypatch, case):
    """MPulse's "fielddiag" writes a file per output step (Ex, every 4 steps,
    "Ex#t.h5") and one appended file (By every 3 steps, "all.h5"); the
    device state dumped at the same steps with the same patterns gives files
    with the same names, dataset names, dims and values (FP64, <= 1e-12)."""
    from oracle import pyoracle
    from tests.cases import make_case, random_fields, rel_l2
    if not os.path.exists(pyoracle.REF_BIN):
        pytest.skip("reference build absent")
    cfg = make_case(case, abi.MP_FP64)
    init = random_fields(cfg, seed=31)
    steps = 9
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    ref_dir.mkdir()
    our_dir.mkdir()
    monkeypatch.setenv("MPULSE_REF_HDF5_LOG", "1")
    diags = (f"fielddiag {{ field Ex file {ref_dir}/Ex#t.h5 interval 4 }} "
             f"fielddiag {{ field By file {ref_dir}/all.h5 interval 3 append y }}")
    pyoracle.run_reference(cfg, steps, init, inits=diags, workdir=str(ref_dir))
    # the same schedule: DiagnosticInterface::execute runs after every step
    # with Process::time = n (the step just taken), a diagnostic's own count
    # from 0 (diagnostic.cpp:12-31)
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        appended = runtime.Hdf5File(f"{our_dir}/all.h5", 0, 0)
        for n in range(steps):
            g.step(1)
            if n % 4 == 0:
                g.write_hdf5(f"{our_dir}/Ex#t.h5", ["Ex"], time=n)
            if n % 3 == 0:
                appended.write_field(g, "By")
        appended.close()
    ref_files = sorted(p.name[:-len(".calls")] for p in ref_dir.glob("*.h5.calls"))
    assert ref_files == ["Ex0.h5", "Ex4.h5", "Ex8.h5", "all.h5"]
    assert sorted(p.name for p in our_dir.glob("*.h5")) == ref_files
    for name in ref_files:
        want = _reference_records(str(ref_dir / name))
        got = read_datasets(str(our_dir / name))
        assert sorted(got) == sorted(want), name
        for ds in want:
            assert got[ds].shape == want[ds].shape == (cfg.nz + 2, cfg.ny + 2, cfg.nx + 2)
            assert rel_l2(got[ds], want[ds]) <= 1e-12, (name, ds)


@pytest.mark.gpu
def test_slices_match_mpulse_slicediag(tmp_path, monkeypatch):
    """MPulse's "slicediag" (FieldSliceDiag) writes a plane of a field per
    output step: Ex in the plane y = 6 every 4 steps to "sy#t.h5", Bz in the
    plane z = 3 every 3 steps appended to one file, and Ey at x = 0 (on the
    boundary: an inactive stream, which creates no file).  The device state
    written with mp_hdf5_write_slice at the same steps gives the same files,
    dataset names, dims and values (FP64, <= 1e-12); the boundary plane gives
    no dataset."""
    from oracle import pyoracle
    from tests.cases import make_case, random_fields, rel_l2
    if not os.path.exists(pyoracle.REF_BIN):
        pytest.skip("reference build absent")
    cfg = make_case("nonlin_all_short", abi.MP_FP64)
    init = random_fields(cfg, seed=37)
    steps = 9
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    ref_dir.mkdir()
    our_dir.mkdir()
    monkeypatch.setenv("MPULSE_REF_HDF5_LOG", "1")
    diags = (f"slicediag {{ field Ex plane y pos 6 file {ref_dir}/sy#t.h5 interval 4 }} "
             f"slicediag {{ field Bz plane z pos 3 file {ref_dir}/sz.h5 interval 3 append y }} "
             f"slicediag {{ field Ey plane x pos 0 file {ref_dir}/sx#t.h5 interval 5 }}")
    pyoracle.run_reference(cfg, steps, init, inits=diags, workdir=str(ref_dir))
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        appended = runtime.Hdf5File(f"{our_dir}/sz.h5", 0, 0)
        for n in range(steps):
            g.step(1)
            if n % 4 == 0:
                with runtime.Hdf5File(f"{our_dir}/sy#t.h5", 0, n) as f:
                    f.write_slice(g, "Ex", "y", 6)
            if n % 3 == 0:
                appended.write_slice(g, "Bz", "z", 3)
        appended.close()
        # the boundary plane: no dataset (MPulse creates no file for it)
        with runtime.Hdf5File(str(tmp_path / "boundary.h5")) as f:
            f.write_slice(g, "Ey", "x", 0)
            f.write_slice(g, "Ey", "x", cfg.nx + 1)
        assert read_datasets(f.name) == {}
    ref_files = sorted(p.name[:-len(".calls")] for p in ref_dir.glob("*.h5.calls"))
    assert ref_files == ["sy0.h5", "sy4.h5", "sy8.h5", "sz.h5"]
    assert sorted(p.name for p in our_dir.glob("*.h5")) == ref_files
    shapes = {"sy": (cfg.nz + 2, cfg.nx + 2), "sz": (cfg.ny + 2, cfg.nx + 2)}
    for name in ref_files:
        want = _reference_records(str(ref_dir / name))
        got = read_datasets(str(our_dir / name))
        assert sorted(got) == sorted(want), name
        for ds in want:
            assert got[ds].shape == want[ds].shape == shapes[name[:2]]
            assert rel_l2(got[ds], want[ds]) <= 1e-12, (name, ds)
    assert sorted(read_datasets(str(our_dir / "sz.h5"))) == ["data0", "data1", "data2"]
