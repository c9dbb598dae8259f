"""Checkpoint files: the reference's restart names and layout
(simulation_data/Time, node_cell_data/Conservatives, ...), written and read
back unchanged."""
import numpy as np
import pytest

from alpaca_b200 import api
from alpaca_b200 import native as N


def test_checkpoint_file_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    ck = {"dim": 2, "t": 0.123456789, "steps": 17, "max_steps": 40, "t_end": 0.5, "cfl": 0.6,
          "cell_size": 1.0 / 64, "gamma": 1.4, "background_pressure": 0.0, "safe": 0,
          "scheme": api.scheme_fields(N.Scheme.make("fsroe", N.FP32_FLUX)),
          "nbr26": rng.integers(-2, 6, (6, 26)).astype(np.int32),
          "blocks": rng.standard_normal((6, 4, 24, 24, 1))}
    path = tmp_path / "case.npz"
    api.save_checkpoint(str(path), ck)
    with np.load(path) as z:
        assert float(z["simulation_data/Time"]) == ck["t"]
        assert int(z["simulation_data/Dimensions"]) == 2
        assert z["node_cell_data/Conservatives"].shape == (6, 4, 24, 24, 1)
    back = api.load_checkpoint(str(path))
    for k, v in ck.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(back[k], v) and back[k].dtype == v.dtype, k
        else:
            assert back[k] == v, k


def test_checkpoint_file_without_scheme_is_rejected(tmp_path):
    """A file that does not record the scheme selection cannot be resumed:
    the case could continue with other numerics."""
    ck = {"dim": 1, "t": 0.0, "steps": 0, "max_steps": 0, "t_end": 1.0, "cfl": 0.6,
          "cell_size": 0.1, "gamma": 1.4, "background_pressure": 0.0, "safe": 0,
          "scheme": api.scheme_fields(N.Scheme.make("fvchar")),
          "nbr26": np.zeros((1, 26), np.int32), "blocks": np.zeros((1, 3, 24, 1, 1))}
    path = str(tmp_path / "case.npz")
    api.save_checkpoint(path, ck)
    with np.load(path) as z:
        kept = {k: z[k] for k in z.files if k != "case/Scheme"}
    np.savez(path, **kept)
    with pytest.raises(ValueError, match="scheme"):
        api.load_checkpoint(path)
