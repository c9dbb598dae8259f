"""Checkpoint files: the reference's restart names and layout
(simulation_data/Time, node_cell_data/Conservatives, ...), written and read
back unchanged."""
import numpy as np

from alpaca_b200 import api


def test_checkpoint_file_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    ck = {"dim": 2, "t": 0.123456789, "steps": 17, "max_steps": 40, "t_end": 0.5, "cfl": 0.6,
          "cell_size": 1.0 / 64, "gamma": 1.4, "background_pressure": 0.0, "safe": 0,
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
