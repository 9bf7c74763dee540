"""The checkpoint format (the reference's fields.npz, utils.py:183-258):
slchannel_b200.utils reads the .npz
the reference's save_flow_fields writes (tests/golden/fields_ckpt.npz, made
by make_checkpoint_golden.py) and writes the same keys, dtypes, shapes and
values; the restart reader re-applies the wall ghosts as the reference's
initialize_flow_from_file does (initflow.py:270-281)."""

import os
import sys

import numpy as np
import pytest
import torch

from slchannel_b200.initflow import initialize_flow_from_file
from slchannel_b200.utils import load_flow_fields, save_flow_fields

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_checkpoint_golden as G  # noqa: E402

GOLD = os.path.join(HERE, "golden", "fields_ckpt.npz")


def test_reads_reference_checkpoint():
    a = G.checkpoint_inputs()
    f = load_flow_fields(GOLD)
    for k in ("u", "v", "w", "p", "z_c", "z_f"):
        assert torch.equal(f[k], torch.from_numpy(a[k]))
    for k in ("Lx", "Ly", "time", "u_tau", "forcing"):
        assert f[k] == a[k] and isinstance(f[k], float)
    assert f["step"] == a["step"] and isinstance(f["step"], int)


def test_writes_reference_format(tmp_path):
    a = G.checkpoint_inputs()
    T = torch.from_numpy
    save_flow_fields(T(a["u"]), T(a["v"]), T(a["w"]), T(a["p"]), T(a["z_c"]), T(a["z_f"]), a["Lx"],
                     a["Ly"], a["step"], a["time"], torch.tensor(a["u_tau"]), a["forcing"],
                     str(tmp_path), "mine.npz")
    mine, ref = np.load(tmp_path / "mine.npz"), np.load(GOLD)
    assert sorted(mine.files) == sorted(ref.files)
    for k in ref.files:
        assert mine[k].dtype == ref[k].dtype and mine[k].shape == ref[k].shape, k
        assert np.array_equal(mine[k], ref[k]), k


def test_restart_reader_reapplies_wall_ghosts():
    u, v, w, p, step, time = initialize_flow_from_file(GOLD)
    assert step == 1234 and time == 12.34
    assert torch.equal(u[:, :, 0], -u[:, :, 1]) and torch.equal(u[:, :, -1], -u[:, :, -2])
    assert torch.equal(v[:, :, 0], -v[:, :, 1]) and torch.equal(v[:, :, -1], -v[:, :, -2])
    assert float(w[:, :, 0].abs().max()) == 0.0 and float(w[:, :, -1].abs().max()) == 0.0
    _, _, _, _, s0, t0 = initialize_flow_from_file(GOLD, reset_time=True)
    assert s0 == 0 and t0 == 0.0


def test_missing_file_raises():
    with pytest.raises(FileNotFoundError):
        load_flow_fields("/nonexistent/fields.npz")
