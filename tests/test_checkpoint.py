"""Restart checkpoints (twophaseflow_b200.checkpoint) on the host: the
reference's ``.npz`` format (src/twophase/simulation/checkpoint.py), its
validation, and a checkpoint the reference's own writer produced
(tests/golden/c1_checkpoint_ref.npz, three quick-start steps, written by
tests/golden/make_golden.py ``checkpoint``).

The solver here is a host-only fake implementing the checkpoint protocol
with NumPy arrays; the GPU step's restore is tested in
tests/test_checkpoint_gpu.py."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from twophaseflow_b200 import checkpoint as ck
from twophaseflow_b200.grid import UniformGrid

HERE = os.path.dirname(__file__)
REF_CKPT = os.path.join(HERE, "golden", "c1_checkpoint_ref.npz")
REF_YAML = os.path.join(HERE, "golden", "c1_checkpoint.yaml")


class HostSolver:
    """The checkpoint protocol over NumPy arrays."""

    backend_device = "cpu"

    def __init__(self, N=(4, 6), seed=0):
        self.grid = UniformGrid(N)
        rng = np.random.default_rng(seed)
        shp = self.grid.shape
        self.p_prev = rng.standard_normal(shp)
        self.conv = [rng.standard_normal(shp) for _ in range(len(N))]
        self.ready = True
        self.contacts = ck.WallContactSet.empty()
        self.restored = None

    def checkpoint_config(self):
        return {"N": list(self.grid.N), "Re": 100.0}

    def checkpoint_state(self):
        return {"p_prev_dev": self.p_prev, "conv_prev": self.conv, "conv_ab2_ready": self.ready,
                "wall_contacts": self.contacts}

    def restore_checkpoint_state(self, st):
        self.restored = st
        return {"psi": st["psi"], "u": st["velocity"][0], "v": st["velocity"][1], "p": st["p"]}


def _fields(shape, seed=1):
    rng = np.random.default_rng(seed)
    return {k: rng.standard_normal(shape) for k in ("psi", "u", "v", "p")}


def _yaml(path, **kw):
    body = {"run": {"T_final": kw.get("t_final", 0.1), "cfl": kw.get("cfl", 0.05), "print_every": 10,
                    "snap_interval": kw.get("snap", 0.05)},
            "grid": {"NX": 4, "NY": 6},
            "output": {"dir": kw.get("out", "results/a")}}
    import yaml
    path.write_text(yaml.safe_dump(body))
    return path


def test_config_fingerprint_ignores_restart_allowed_entries(tmp_path):
    a = _yaml(tmp_path / "a.yaml")
    b = _yaml(tmp_path / "b.yaml", t_final=0.7, snap=0.01, out="results/other")
    c = _yaml(tmp_path / "c.yaml", cfl=0.08)
    assert ck.config_fingerprint(a) == ck.config_fingerprint(b)
    assert ck.config_fingerprint(a) != ck.config_fingerprint(c)
    nested = tmp_path / "n.yaml"
    nested.write_text("run:\n  time:\n    final: 1.0\n    cfl: 0.2\n    print_every: 5\noutput:\n  dir: x\n")
    nested2 = tmp_path / "n2.yaml"
    nested2.write_text("run:\n  time:\n    final: 3.0\n    cfl: 0.2\n    print_every: 50\noutput:\n  dir: y\n")
    assert ck.config_fingerprint(nested) == ck.config_fingerprint(nested2)


def test_roundtrip_restores_history_and_outputs(tmp_path):
    cfg = _yaml(tmp_path / "cfg.yaml")
    s = HostSolver()
    f = _fields(s.grid.shape)
    s.contacts = ck.WallContactSet(
        contacts=(ck.WallContact(0, "lo", 1, float(np.pi / 7.0), -1.0, "pinned_no_slip", "mirror_neutral", 0.5),),
        traces=(ck.WallTrace(0, "hi", 1, (0.0, 0.5, 1.0), (0.1, float(np.pi / 9.0), 0.9), 0.5),))
    path = tmp_path / "checkpoint_final.npz"
    ck.save_checkpoint(path, solver=s, **f, t=0.125, step=5, config_path=cfg,
                       results={"times": np.array([0.0, 0.125]), "label": "skipped (not an array)"},
                       snapshots=[{"t": 0.0, "psi": f["psi"], "pressure_accel_faces": [np.ones((3, 6)), np.ones((4, 5))]},
                                  {"t": 0.125, "psi": 2 * f["psi"], "psi_after_reinit": f["psi"],
                                   "pressure_accel_faces": [np.zeros((3, 6)), np.zeros((4, 5))]}],
                       debug_history=[{"kappa_max": 1.0, "it": 3}, {"kappa_max": 2.0, "it": 4}],
                       state_phase="pre_step", dt_candidate=0.01, dt_effective=0.004, terminal_clamped=True)
    assert ck.default_checkpoint_path(tmp_path) == path
    r = HostSolver(seed=9)
    st = ck.load_checkpoint(path, solver=r, config_path=cfg)
    assert (st["t"], st["step"], st["state_phase"]) == (0.125, 5, "pre_step")
    assert (st["dt_candidate"], st["dt_effective"], st["terminal_clamped"]) == (0.01, 0.004, True)
    for k in ("psi", "u", "v", "p"):
        np.testing.assert_array_equal(st[k], f[k])
    got = r.restored
    np.testing.assert_array_equal(got["p_prev_dev"], s.p_prev)
    for a, b in zip(got["conv_prev"], s.conv):
        np.testing.assert_array_equal(a, b)
    assert got["conv_ab2_ready"] is True and got["velocity_bdf2_ready"] is False
    assert got["velocity_prev"] is None and got["p_base_prev_dev"] is None
    c = got["wall_contacts"].contacts[0]
    assert np.float64(c.coordinate).tobytes() == np.float64(np.pi / 7.0).tobytes()
    assert c.angle_mode == "mirror_neutral"
    t = got["wall_contacts"].traces[0]
    assert t.wall_side == "hi" and np.float64(t.values[1]).tobytes() == np.float64(np.pi / 9.0).tobytes()
    assert list(st["results"]) == ["times"]
    assert [snap["t"] for snap in st["snapshots"]] == [0.0, 0.125]
    np.testing.assert_array_equal(st["snapshots"][1]["psi"], 2 * f["psi"])
    assert "psi_after_reinit" not in st["snapshots"][1]        # not present in every snapshot
    assert st["snapshots"][0]["pressure_accel_faces"][1].shape == (4, 5)
    assert st["debug_history"] == [{"kappa_max": 1.0, "it": 3}, {"kappa_max": 2.0, "it": 4}]
    m = ck.load_manifest(path)
    assert m["magic"] == ck.MAGIC and m["schema_version"] == ck.SCHEMA_VERSION and m["grid_shape"] == [5, 7]


def test_options_fingerprint_without_config_file(tmp_path):
    s = HostSolver()
    path = tmp_path / "c.npz"
    ck.save_checkpoint(path, solver=s, **_fields(s.grid.shape), t=0.0, step=0)
    ck.load_checkpoint(path, solver=HostSolver(), config_path=None)
    other = HostSolver()
    other.checkpoint_config = lambda: {"N": [4, 6], "Re": 200.0}
    with pytest.raises(ck.CheckpointError, match="config fingerprint"):
        ck.load_checkpoint(path, solver=other)


def test_validation_rejects(tmp_path, monkeypatch):
    cfg = _yaml(tmp_path / "cfg.yaml")
    s = HostSolver()
    f = _fields(s.grid.shape)
    path = tmp_path / "c.npz"
    ck.save_checkpoint(path, solver=s, **f, t=0.1, step=1, config_path=cfg)
    with pytest.raises(ck.CheckpointError, match="config fingerprint"):
        ck.load_checkpoint(path, solver=HostSolver(), config_path=_yaml(tmp_path / "d.yaml", cfl=0.5))
    with pytest.raises(ck.CheckpointError, match="grid shape"):
        ck.load_checkpoint(path, solver=HostSolver(N=(4, 4)), config_path=cfg)
    with pytest.raises(ck.CheckpointError, match="state_phase"):
        ck.save_checkpoint(path, solver=s, **f, t=0.1, step=1, config_path=cfg, state_phase="mid_step")
    monkeypatch.setattr(ck, "code_fingerprint", lambda package_root=None: "0" * 64)
    with pytest.raises(ck.CheckpointError, match="code fingerprint"):
        ck.load_checkpoint(path, solver=HostSolver(), config_path=cfg)
    ck.load_checkpoint(path, solver=HostSolver(), config_path=cfg, verify_code=False)
    monkeypatch.undo()
    # tampered payload, magic and missing state arrays
    with np.load(path) as d:
        arrays = {k: d[k] for k in d.files}
    bad = dict(arrays)
    bad["state/u"] = bad["state/u"] + 1.0
    np.savez(tmp_path / "t.npz", **bad)
    with pytest.raises(ck.CheckpointError, match="payload hash"):
        ck.load_checkpoint(tmp_path / "t.npz", solver=HostSolver(), config_path=cfg)
    man = json.loads(arrays["__manifest_json__"].tobytes())
    man["magic"] = "other"
    bad = dict(arrays)
    bad["__manifest_json__"] = np.frombuffer(json.dumps(man).encode(), dtype=np.uint8)
    np.savez(tmp_path / "m.npz", **bad)
    with pytest.raises(ck.CheckpointError, match="magic"):
        ck.load_checkpoint(tmp_path / "m.npz", solver=HostSolver(), config_path=cfg)
    bad = {k: v for k, v in arrays.items() if k != "state/p"}
    np.savez(tmp_path / "p.npz", **bad)
    with pytest.raises(ck.CheckpointError, match="missing required array state/p"):
        ck.load_checkpoint(tmp_path / "p.npz", solver=HostSolver(), config_path=cfg)


def test_atomic_write_leaves_no_temporary(tmp_path):
    s = HostSolver()
    path = tmp_path / "sub" / "checkpoint_final.npz"
    for step in range(3):
        ck.save_checkpoint(path, solver=s, **_fields(s.grid.shape, seed=step), t=float(step), step=step)
    assert sorted(os.listdir(path.parent)) == ["checkpoint_final.npz"]
    assert ck.load_manifest(path)["step"] == 2


def test_reference_written_checkpoint_validates_and_decodes():
    """The reference's writer and this loader agree on every hash and key:
    the payload and grid hashes validate, the config fingerprint of the
    committed YAML matches, and only the code fingerprint (the reference's
    tree) differs."""
    g = np.load(os.path.join(HERE, "golden", "c1_golden.npz"))
    s = HostSolver(N=(64, 64))
    with pytest.raises(ck.CheckpointError, match="code fingerprint"):
        ck.load_checkpoint(REF_CKPT, solver=s, config_path=REF_YAML)
    st = ck.load_checkpoint(REF_CKPT, solver=s, config_path=REF_YAML, verify_code=False)
    assert st["step"] == 3 and st["state_phase"] == "post_step"
    for f in ("psi", "u", "v", "p"):
        np.testing.assert_array_equal(st[f], g[f"s2/{f}"])
    got = s.restored
    assert got["conv_ab2_ready"] is True and len(got["conv_prev"]) == 2
    np.testing.assert_array_equal(got["p_prev_dev"], g["s2/p"])
    np.testing.assert_array_equal(got["grid_coords"][0], np.linspace(0.0, 1.0, 65))
    assert st["dt_effective"] == float(g["s2/dt"])
    assert abs(st["t"] - float(g["s0/dt"] + g["s1/dt"] + g["s2/dt"])) <= 1e-18


def test_this_writer_loads_in_the_reference(tmp_path, monkeypatch):
    """A checkpoint this package wrote restores through the reference's own
    load_checkpoint (code fingerprint bypassed: it hashes the reference's
    tree).  Runs where the reference source is importable."""
    src = os.environ.get("TWOPHASE_REFERENCE_SRC", "/root/reference/src")
    if not os.path.isdir(os.path.join(src, "twophase")):
        pytest.skip("reference source not present")
    import sys
    from types import SimpleNamespace
    monkeypatch.syspath_prepend(src)
    monkeypatch.setattr(sys, "dont_write_bytecode", True)   # the reference tree is read-only
    try:
        import twophase.simulation.checkpoint as rck
    except Exception as e:  # pragma: no cover - dependency gaps in the reference
        pytest.skip(f"reference checkpoint module not importable: {e}")
    cfg = _yaml(tmp_path / "cfg.yaml")
    s = HostSolver()
    f = _fields(s.grid.shape)
    path = tmp_path / "c.npz"
    ck.save_checkpoint(path, solver=s, **f, t=0.25, step=7, config_path=cfg)
    monkeypatch.setattr(rck, "code_fingerprint", lambda root: ck.load_manifest(path)["code_fingerprint"])

    class _G:
        ndim, shape, N, L = 2, s.grid.shape, s.grid.N, s.grid.L

        def __init__(self):
            self.coords = [np.zeros(n) for n in self.shape]
            self.h = [np.zeros(n) for n in self.shape]

        def _build_metrics(self, ccd=None):
            pass

        def meshgrid(self):
            return np.meshgrid(*self.coords, indexing="ij")

    aware = SimpleNamespace(update_grid=lambda g: None, invalidate_cache=lambda: None, update_weights=lambda: None)
    rs = SimpleNamespace(_backend=SimpleNamespace(xp=np, to_host=lambda a: a), _grid=_G(), _ccd=None, _reinit=aware,
                         _ppe_solver=aware, _fccd_div_op=None)
    rs.set_wall_contacts = lambda c: setattr(rs, "_wall_contacts", c)
    st = rck.load_checkpoint(path, solver=rs, config_path=cfg)
    assert st["step"] == 7 and st["t"] == 0.25
    np.testing.assert_array_equal(st["u"], f["u"])
    np.testing.assert_array_equal(rs._grid.coords[1], s.grid.coords[1])
    np.testing.assert_array_equal(rs._p_prev_dev, s.p_prev)
    np.testing.assert_array_equal(rs._conv_prev[1], s.conv[1])
    assert rs._conv_ab2_ready is True
