"""The statistics restart format (turbstats.py:464-609), on CPU: the drop-in's
TurbulenceStats.load_state reads the state the reference's save_state wrote
(tests/golden/stats_state.npz, from make_stats_golden.py), its save_state
writes the same keys, in the same order, with the same values, and its
error and compatibility paths behave as the reference's do.

The state methods touch only the accumulators and counters, so they run here
on a stand-in that holds those as CPU tensors (the class itself allocates
them on the GPU)."""

import os
import shutil
import sys

import numpy as np
import pytest
import torch

from slchannel_b200.turbstats import PROFILES, SPECTRA, TurbulenceStats

HERE = os.path.dirname(__file__)
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_stats_golden import EXTRA_PLANES, N_SNAPSHOTS, NX, NY, NZ  # noqa: E402

STATE = os.path.join(HERE, "golden", "stats_state.npz")
FINAL = os.path.join(HERE, "golden", "stats_final.npz")
KINDS = ("uu", "vv", "ww", "uw")


class Accumulators:
    """The attributes TurbulenceStats' state I/O reads and writes, on CPU."""

    def __init__(self, nx=NX, ny=NY, nz=NZ, planes=EXTRA_PLANES):
        f = dict(dtype=torch.float64)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n_samples = 0
        for name in PROFILES:
            setattr(self, name, torch.zeros(nz, **f))
        for name in SPECTRA:
            setattr(self, name, torch.zeros(nx // 2, ny // 2, **f))
        self.spectra_z_planes = [float(p) for p in planes]
        self.n_samples_extra = 0
        self.extra_planes = [{"zp": zp, "sums": {k: torch.zeros(nx // 2, ny // 2, **f) for k in KINDS}}
                             for zp in self.spectra_z_planes]


def _load(acc, path):
    TurbulenceStats.load_state(acc, path)
    return acc


def test_reads_the_reference_state():
    ref = np.load(STATE)
    acc = _load(Accumulators(), STATE)
    assert acc.n_samples == N_SNAPSHOTS and acc.n_samples_extra == N_SNAPSHOTS
    for name in PROFILES + SPECTRA:
        np.testing.assert_array_equal(getattr(acc, name).numpy(), ref[name], err_msg=name)
    for pl in acc.extra_planes:
        for k in KINDS:
            np.testing.assert_array_equal(pl["sums"][k].numpy(), ref[f"E_{k}_2d_z{pl['zp']:.0f}_sum"])


def test_writes_the_reference_layout(tmp_path):
    acc = _load(Accumulators(), STATE)
    out = tmp_path / "state.npz"
    TurbulenceStats.save_state(acc, str(out))
    ref, got = np.load(STATE), np.load(out)
    assert got.files == ref.files
    for key in ref.files:
        assert got[key].dtype == ref[key].dtype, key
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)


def test_restart_round_trip_continues_the_counts(tmp_path):
    acc = _load(Accumulators(), STATE)
    acc.U_sum += 1.0
    acc.n_samples += 1
    out = tmp_path / "state.npz"
    TurbulenceStats.save_state(acc, str(out))
    again = _load(Accumulators(), str(out))
    assert again.n_samples == N_SNAPSHOTS + 1
    np.testing.assert_array_equal(again.U_sum.numpy(), np.load(STATE)["U_sum"] + 1.0)


def test_grid_mismatch_is_refused():
    with pytest.raises(ValueError, match=r"Grid dimension mismatch! State file has \(nx=8, ny=6, nz=12\)"):
        _load(Accumulators(nz=NZ + 2), STATE)


def test_missing_files_raise():
    with pytest.raises(FileNotFoundError, match="Statistics state file not found"):
        _load(Accumulators(), "/nonexistent/stats_state.npz")
    with pytest.raises(FileNotFoundError, match="Statistics file not found"):
        TurbulenceStats.load_statistics("/nonexistent/stats.npz")


def test_other_plane_set_starts_the_extra_planes_fresh():
    ref = np.load(STATE)
    acc = _load(Accumulators(planes=[50.0]), STATE)
    assert acc.n_samples == N_SNAPSHOTS and acc.n_samples_extra == 0
    np.testing.assert_array_equal(acc.U_sum.numpy(), ref["U_sum"])
    assert all(float(t.abs().sum()) == 0.0 for t in acc.extra_planes[0]["sums"].values())


def test_state_without_plane_mean_moments_warns(tmp_path):
    ref = np.load(STATE)
    old = {k: ref[k] for k in ref.files
           if k not in ("Vm_sum", "Wm_sum", "Um2_sum", "Vm2_sum", "Wm2_sum", "UmWm_sum")}
    path = tmp_path / "old_state.npz"
    np.savez_compressed(path, **old)
    with pytest.warns(RuntimeWarning, match="plane-mean moments"):
        acc = _load(Accumulators(), str(path))
    np.testing.assert_array_equal(acc.uu_sum.numpy(), ref["uu_sum"])
    assert float(acc.Um2_sum.abs().sum()) == 0.0


def test_wrong_array_shape_is_refused(tmp_path):
    ref = np.load(STATE)
    bad = {k: ref[k] for k in ref.files}
    bad["U_sum"] = np.zeros(NZ + 1)
    path = tmp_path / "bad_state.npz"
    np.savez_compressed(path, **bad)
    with pytest.raises(ValueError, match="U_sum: shape"):
        _load(Accumulators(), str(path))


def test_load_statistics_reads_the_reference_file(tmp_path):
    got = TurbulenceStats.load_statistics(FINAL)
    ref = np.load(FINAL)
    assert sorted(got) == sorted(ref.files)
    for key in ref.files:
        np.testing.assert_array_equal(got[key], ref[key])
    copy = tmp_path / "copy.npz"
    shutil.copy(FINAL, copy)
    assert sorted(TurbulenceStats.load_statistics(str(copy))) == sorted(ref.files)
