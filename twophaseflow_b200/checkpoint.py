"""Restart checkpoints in the reference's ``.npz`` format.

Mirrors ``twophase.simulation.checkpoint`` (src/twophase/simulation/
checkpoint.py:88-237, schema 2): one compressed ``.npz`` written by an atomic
replace, holding

* ``state/psi``, ``state/u``, ``state/v``, ``state/p`` (and ``state/w`` for a
  3-D run, which the reference's 2-D solver never writes);
* ``grid/coords/<axis>``, ``grid/h/<axis>``;
* the solver history the next step reads: ``solver/p_prev_dev``,
  ``solver/conv_prev/{count,<i>}`` (the AB2 convection history),
  ``solver/velocity_prev``, ``solver/p_prev_accel_face_components``,
  ``solver/projected_face_components``,
  ``solver/conservative_momentum_components`` (each ``count`` 0 when the
  pipeline keeps none), ``solver/flags`` = [AB2 ready, BDF2 ready] and the
  wall-contact arrays (``solver/wall_contacts/contacts`` (k, 8) float64,
  ``trace_count`` and per-trace arrays);
* ``results/*``, ``snapshots/*`` and ``debug/*`` when given;
* ``__manifest_json__``: the JSON manifest as uint8 bytes (magic, schema,
  time, step, state phase, dt candidate / effective, grid shape, SHA-256 of
  the grid arrays and of the whole payload, the config fingerprint and the
  code fingerprint).

The key names, array encodings, manifest fields and validation messages are
the reference's, so a checkpoint either side writes carries the same state
under the same names.  Two differences, both about identity rather than
state:

* ``code_fingerprint`` hashes this package's sources (Python, CUDA, headers),
  not the reference's tree and git HEAD; ``load_checkpoint(...,
  verify_code=False)`` accepts a checkpoint another code base wrote (the
  reference's own, for instance) while keeping every other check.
* ``config_path`` may be None for a solver built from keyword options; the
  config fingerprint is then the hash of ``solver.checkpoint_config()``.

The solver protocol: ``grid`` (``ndim``, ``shape``, ``coords``, ``h``),
``checkpoint_state()`` returning the named history (``p_prev_dev``,
``conv_prev``, ``conv_ab2_ready`` ...), ``restore_checkpoint_state(state)``,
``checkpoint_config()`` and ``backend_device``.  ``TwoPhaseStep`` implements
it; arrays may be torch tensors on the device or NumPy arrays, and everything
on disk is host NumPy.
"""

from __future__ import annotations

import hashlib
import json
import os
import pathlib
import tempfile
from dataclasses import dataclass
from typing import Any

import numpy as np

SCHEMA_VERSION = 2
SUPPORTED_SCHEMA_VERSIONS = (1, 2)
MAGIC = "twophase.ch14.restart"
CHECKPOINT_STATE_PHASES = ("pre_step", "post_step")
# config entries that may change between a run and its restart
# (the reference's list, checkpoint.py:47-59)
RESTART_ALLOWED_CONFIG_PATHS = (
    ("run", "T_final"),
    ("run", "time", "final"),
    ("run", "snap_times"),
    ("run", "snapshots", "times"),
    ("run", "snap_interval"),
    ("run", "snapshots", "interval"),
    ("run", "print_every"),
    ("run", "time", "print_every"),
    ("run", "debug_diagnostics"),
    ("run", "debug", "step_diagnostics"),
    ("output",),
)
SNAPSHOT_FIELDS = ("psi", "u", "v", "p", "rho", "psi_before_transport", "psi_after_transport_before_reinit",
                   "psi_after_reinit", "geometric_q", "geometric_phi", "geometric_density")
# history lists the reference's solver may hold; the B200 step keeps conv_prev
HISTORY_LISTS = ("p_prev_accel_face_components", "conv_prev", "velocity_prev", "projected_face_components",
                 "conservative_momentum_components")
HISTORY_ARRAYS = ("p_prev_dev", "p_base_prev_dev", "p_base_prev2_dev", "conservative_density")
WALL_SIDES = ("lo", "hi")
CONTACT_MODES = ("pinned_no_slip",)
ANGLE_MODES = ("initial", "mirror_neutral", "unspecified")
_SOURCE_SUFFIXES = (".py", ".cu", ".cuh", ".h", ".cpp")


class CheckpointError(RuntimeError):
    """A checkpoint failed validation (format, identity, or shape)."""


@dataclass(frozen=True)
class WallContact:
    wall_axis: int
    wall_side: str
    tangent_axis: int
    coordinate: float
    orientation: float
    mode: str = "pinned_no_slip"
    angle_mode: str = "initial"
    level: float = 0.5


@dataclass(frozen=True)
class WallTrace:
    wall_axis: int
    wall_side: str
    tangent_axis: int
    tangent_coordinates: tuple
    values: tuple
    level: float = 0.5


@dataclass(frozen=True)
class WallContactSet:
    contacts: tuple = ()
    traces: tuple = ()

    @classmethod
    def empty(cls):
        return cls()


def default_checkpoint_path(outdir) -> pathlib.Path:
    """``<outdir>/checkpoint_final.npz``."""
    return pathlib.Path(outdir) / "checkpoint_final.npz"


# -- host conversion -------------------------------------------------------------
def _host(value) -> np.ndarray:
    if hasattr(value, "detach"):          # torch tensor, any device
        return value.detach().cpu().numpy().copy()
    return np.array(value, copy=True)


def _json_bytes(payload) -> np.ndarray:
    raw = json.dumps(payload, sort_keys=True, separators=(",", ":")).encode("utf-8")
    return np.frombuffer(raw, dtype=np.uint8).copy()


def _from_json_bytes(value):
    return json.loads(np.asarray(value, dtype=np.uint8).tobytes().decode("utf-8"))


def _sha256_arrays(arrays: dict, select=None) -> str:
    d = hashlib.sha256()
    for key in sorted(arrays):
        if select is not None and not select(key):
            continue
        a = np.asarray(arrays[key])
        d.update(key.encode("utf-8"))
        d.update(str(a.shape).encode("ascii"))
        d.update(str(a.dtype).encode("ascii"))
        d.update(np.ascontiguousarray(a).tobytes())
    return d.hexdigest()


def _grid_hash(arrays: dict) -> str:
    return _sha256_arrays(arrays, lambda k: k.startswith("grid/coords/") or k.startswith("grid/h/"))


def _payload_hash(arrays: dict) -> str:
    return _sha256_arrays(arrays)


# -- fingerprints ------------------------------------------------------------------
def _without_paths(raw, paths):
    data = json.loads(json.dumps(raw, default=str))
    for path in paths:
        node = data
        for key in path[:-1]:
            node = node.get(key) if isinstance(node, dict) else None
            if node is None:
                break
        if isinstance(node, dict):
            node.pop(path[-1], None)
    return data


def config_fingerprint(config_path) -> str:
    """SHA-256 of the YAML config with the restart-allowed entries removed."""
    import yaml
    with open(config_path) as fh:
        raw = yaml.safe_load(fh) or {}
    canon = json.dumps(_without_paths(raw, RESTART_ALLOWED_CONFIG_PATHS), sort_keys=True, separators=(",", ":"),
                       default=str)
    return hashlib.sha256(canon.encode("utf-8")).hexdigest()


def _options_fingerprint(options: dict) -> str:
    canon = json.dumps(options, sort_keys=True, separators=(",", ":"), default=str)
    return hashlib.sha256(canon.encode("utf-8")).hexdigest()


def code_fingerprint(package_root=None) -> str:
    """SHA-256 over this package's source files (relative path + bytes)."""
    root = pathlib.Path(package_root) if package_root is not None else pathlib.Path(__file__).resolve().parent
    files = sorted(p for p in root.rglob("*") if p.is_file() and p.suffix in _SOURCE_SUFFIXES
                   and "__pycache__" not in p.parts)
    d = hashlib.sha256()
    for p in files:
        d.update(p.relative_to(root).as_posix().encode("utf-8"))
        d.update(p.read_bytes())
    return d.hexdigest()


def _solver_config_hash(solver, config_path):
    if config_path is not None:
        return config_fingerprint(config_path)
    cfg = getattr(solver, "checkpoint_config", None)
    if not callable(cfg):
        raise CheckpointError("config_path is None and the solver has no checkpoint_config()")
    return _options_fingerprint(cfg())


# -- capture -----------------------------------------------------------------------
def _capture_grid(arrays, grid):
    for a, c in enumerate(grid.coords):
        arrays[f"grid/coords/{a}"] = np.array(c, dtype=np.float64, copy=True)
    hs = getattr(grid, "h", None)
    if hs is None:
        hs = [np.full(len(c), float(grid.L[a]) / float(grid.N[a])) for a, c in enumerate(grid.coords)]
    for a, h in enumerate(hs):
        arrays[f"grid/h/{a}"] = np.array(h, dtype=np.float64, copy=True)


def _capture_contacts(arrays, contacts):
    contacts = contacts if contacts is not None else WallContactSet.empty()
    rows = [[int(c.wall_axis), WALL_SIDES.index(c.wall_side), int(c.tangent_axis), float(c.coordinate),
             float(c.orientation), CONTACT_MODES.index(c.mode), ANGLE_MODES.index(c.angle_mode), float(c.level)]
            for c in contacts.contacts]
    arrays["solver/wall_contacts/contacts"] = np.asarray(rows, dtype=np.float64)   # shape (0,) when empty
    arrays["solver/wall_contacts/trace_count"] = np.asarray(len(contacts.traces), dtype=np.int64)
    for i, t in enumerate(contacts.traces):
        base = f"solver/wall_contacts/traces/{i}"
        arrays[f"{base}/meta"] = np.asarray([int(t.wall_axis), WALL_SIDES.index(t.wall_side), int(t.tangent_axis),
                                            float(t.level)], dtype=np.float64)
        arrays[f"{base}/tangent_coordinates"] = np.asarray(t.tangent_coordinates, dtype=np.float64)
        arrays[f"{base}/values"] = np.asarray(t.values, dtype=np.float64)


def _capture_solver(arrays, solver):
    st = dict(solver.checkpoint_state())
    if "geometric_phase" in st and st["geometric_phase"] is not None:
        raise CheckpointError("geometric phase state is not carried by this package's checkpoints")
    _capture_grid(arrays, solver.grid)
    for name in HISTORY_ARRAYS:
        if st.get(name) is not None:
            arrays[f"solver/{name}"] = _host(st[name])
    for name in HISTORY_LISTS:
        values = st.get(name)
        arrays[f"solver/{name}/count"] = np.asarray(0 if values is None else len(values), dtype=np.int64)
        for i, v in enumerate(values or ()):
            arrays[f"solver/{name}/{i}"] = _host(v)
    arrays["solver/flags"] = np.asarray([bool(st.get("conv_ab2_ready", False)),
                                         bool(st.get("velocity_bdf2_ready", False))], dtype=bool)
    _capture_contacts(arrays, st.get("wall_contacts"))
    if st.get("reinit_reference_monitor") is not None:
        arrays["solver/transport/reinit_reference_monitor"] = np.asarray(float(st["reinit_reference_monitor"]),
                                                                         dtype=np.float64)


def _capture_outputs(arrays, results, snapshots, debug_history):
    for k, v in (results or {}).items():
        if isinstance(v, np.ndarray):
            arrays[f"results/{k}"] = np.asarray(v)
    if debug_history:
        keys = sorted(debug_history[0])
        arrays["debug/keys_json"] = _json_bytes(keys)
        for k in keys:
            arrays[f"debug/{k}"] = np.asarray([e[k] for e in debug_history])
    if snapshots:
        arrays["snapshots/times"] = np.asarray([s["t"] for s in snapshots], dtype=float)
        for f in SNAPSHOT_FIELDS:
            if all(f in s for s in snapshots):
                arrays[f"snapshots/{f}"] = np.stack([_host(s[f]) for s in snapshots], axis=0)
        for f in ("pressure_accel_faces", "grid_coords"):
            if all(f in s for s in snapshots):
                for a in range(len(snapshots[0][f])):
                    arrays[f"snapshots/{f}/{a}"] = np.stack([_host(s[f][a]) for s in snapshots], axis=0)


def capture_checkpoint_frame(*, solver, psi, u, v, p, t: float, step: int, config_path=None, results=None,
                             snapshots=None, debug_history=None, state_phase: str = "post_step",
                             dt_candidate=None, dt_effective=None, terminal_clamped: bool = False, w=None):
    """The arrays and manifest of a checkpoint, without writing them
    (checkpoint.py:130-187).  ``state_phase='pre_step'`` marks the input of
    the next step rather than the output of the last one."""
    phase = str(state_phase).strip().lower()
    if phase not in CHECKPOINT_STATE_PHASES:
        raise CheckpointError(f"checkpoint state_phase must be one of {CHECKPOINT_STATE_PHASES}, got {state_phase!r}")
    arrays = {"state/psi": _host(psi), "state/u": _host(u), "state/v": _host(v), "state/p": _host(p)}
    if w is not None:
        arrays["state/w"] = _host(w)
    _capture_solver(arrays, solver)
    _capture_outputs(arrays, results, snapshots, debug_history)
    cfg_path = None if config_path is None else str(pathlib.Path(config_path).resolve())
    manifest = {
        "magic": MAGIC,
        "schema_version": SCHEMA_VERSION,
        "time": float(t),
        "step": int(step),
        "state_phase": phase,
        "dt_candidate": None if dt_candidate is None else float(dt_candidate),
        "dt_effective": None if dt_effective is None else float(dt_effective),
        "terminal_clamped": bool(terminal_clamped),
        "backend_device": getattr(solver, "backend_device", "unknown"),
        "grid_shape": [int(n) for n in solver.grid.shape],
        "grid_hash": _grid_hash(arrays),
        "config_path": cfg_path,
        "config_hash_excluding_restart_allowed_paths": _solver_config_hash(solver, config_path),
        "code_fingerprint": code_fingerprint(),
        "payload_hash": _payload_hash(arrays),
    }
    return {"arrays": arrays, "manifest": manifest}


def write_checkpoint_frame(path, frame) -> None:
    """Write a captured frame: temporary file in the target directory, then
    an atomic rename over ``path``."""
    path = pathlib.Path(path)
    arrays = {k: np.asarray(v) for k, v in dict(frame["arrays"]).items()}
    arrays["__manifest_json__"] = _json_bytes(frame["manifest"])
    path.parent.mkdir(parents=True, exist_ok=True)
    fd, tmp = tempfile.mkstemp(prefix=f".{path.name}.", suffix=".tmp", dir=path.parent)
    try:
        with os.fdopen(fd, "wb") as fh:
            np.savez_compressed(fh, **arrays)
        os.replace(tmp, path)
    finally:
        if os.path.exists(tmp):
            os.unlink(tmp)


def save_checkpoint(path, *, solver, psi, u, v, p, t: float, step: int, config_path=None, results=None,
                    snapshots=None, debug_history=None, state_phase: str = "post_step", dt_candidate=None,
                    dt_effective=None, terminal_clamped: bool = False, w=None) -> None:
    """Persist the restart state (checkpoint.py:88-127); device arrays are
    copied to the host, so the file holds plain NumPy arrays."""
    frame = capture_checkpoint_frame(solver=solver, psi=psi, u=u, v=v, p=p, t=t, step=step, config_path=config_path,
                                     results=results, snapshots=snapshots, debug_history=debug_history,
                                     state_phase=state_phase, dt_candidate=dt_candidate, dt_effective=dt_effective,
                                     terminal_clamped=terminal_clamped, w=w)
    write_checkpoint_frame(path, frame)


# -- load --------------------------------------------------------------------------
def load_manifest(path) -> dict:
    """The manifest alone."""
    with np.load(path, allow_pickle=False) as data:
        return _from_json_bytes(data["__manifest_json__"])


def _validate(manifest, arrays, solver, config_path, verify_code):
    if manifest.get("magic") != MAGIC:
        raise CheckpointError("checkpoint magic does not match ch14 restart format")
    if manifest.get("schema_version") not in SUPPORTED_SCHEMA_VERSIONS:
        raise CheckpointError(f"unsupported checkpoint schema {manifest.get('schema_version')}")
    phase = manifest.get("state_phase", "post_step")
    if phase not in CHECKPOINT_STATE_PHASES:
        raise CheckpointError(f"unsupported checkpoint state_phase {phase!r}")
    stored_cfg = manifest.get("config_hash_excluding_restart_allowed_paths",
                              manifest.get("config_hash_excluding_final_time"))
    if stored_cfg != _solver_config_hash(solver, config_path):
        raise CheckpointError("checkpoint config fingerprint differs; only final time and "
                              "visualization/output paths may change")
    if verify_code and manifest.get("code_fingerprint") != code_fingerprint():
        raise CheckpointError("checkpoint code fingerprint differs; refusing restart")
    shape = tuple(int(n) for n in solver.grid.shape)
    if tuple(manifest.get("grid_shape", ())) != shape:
        raise CheckpointError("checkpoint grid shape differs from current config")
    required = ["state/psi", "state/u", "state/v", "state/p"] + (["state/w"] if len(shape) == 3 else [])
    for key in required:
        if key not in arrays:
            raise CheckpointError(f"checkpoint missing required array {key}")
        if tuple(arrays[key].shape) != shape:
            raise CheckpointError(f"checkpoint array {key} shape mismatch")
    if "grid_hash" in manifest and manifest["grid_hash"] != _grid_hash(arrays):
        raise CheckpointError("checkpoint grid hash mismatch")
    if manifest.get("payload_hash") != _payload_hash(arrays):
        raise CheckpointError("checkpoint payload hash mismatch")


def _restore_contacts(arrays) -> WallContactSet:
    rows = np.asarray(arrays.get("solver/wall_contacts/contacts", np.empty((0, 8))), dtype=np.float64).reshape(-1, 8)
    contacts = tuple(WallContact(int(r[0]), WALL_SIDES[int(r[1])], int(r[2]), float(r[3]), float(r[4]),
                                 CONTACT_MODES[int(r[5])], ANGLE_MODES[int(r[6])], float(r[7])) for r in rows)
    traces = []
    for i in range(int(arrays.get("solver/wall_contacts/trace_count", np.asarray(0)))):
        base = f"solver/wall_contacts/traces/{i}"
        m = arrays[f"{base}/meta"]
        traces.append(WallTrace(int(m[0]), WALL_SIDES[int(m[1])], int(m[2]),
                                tuple(float(x) for x in arrays[f"{base}/tangent_coordinates"]),
                                tuple(float(x) for x in arrays[f"{base}/values"]), float(m[3])))
    return WallContactSet(contacts=contacts, traces=tuple(traces))


def _restore_state_dict(arrays) -> dict:
    st: dict[str, Any] = {"psi": arrays["state/psi"], "p": arrays["state/p"],
                          "velocity": [arrays["state/u"], arrays["state/v"]] + (
                              [arrays["state/w"]] if "state/w" in arrays else [])}
    st["grid_coords"] = [arrays[f"grid/coords/{a}"] for a in range(len(st["velocity"])) if f"grid/coords/{a}" in arrays]
    st["grid_h"] = [arrays[f"grid/h/{a}"] for a in range(len(st["velocity"])) if f"grid/h/{a}" in arrays]
    for name in HISTORY_ARRAYS:
        st[name] = arrays.get(f"solver/{name}")
    for name in HISTORY_LISTS:
        n = int(arrays.get(f"solver/{name}/count", np.asarray(0)))
        st[name] = None if n == 0 else [arrays[f"solver/{name}/{i}"] for i in range(n)]
    flags = arrays.get("solver/flags", np.asarray([False, False]))
    st["conv_ab2_ready"] = bool(flags[0])
    st["velocity_bdf2_ready"] = bool(flags[1])
    st["wall_contacts"] = _restore_contacts(arrays)
    key = "solver/transport/reinit_reference_monitor"
    st["reinit_reference_monitor"] = float(arrays[key]) if key in arrays else None
    st["geometric_phase"] = any(k.startswith("solver/geometric_phase/") for k in arrays)
    return st


def _restore_outputs(arrays):
    results = {k[len("results/"):]: v for k, v in arrays.items() if k.startswith("results/")}
    snapshots = []
    if "snapshots/times" in arrays:
        times = arrays["snapshots/times"]

        def series(prefix):
            out, a = [], 0
            while f"{prefix}/{a}" in arrays:
                out.append(arrays[f"{prefix}/{a}"])
                a += 1
            return out
        faces, coords = series("snapshots/pressure_accel_faces"), series("snapshots/grid_coords")
        for i, t in enumerate(times):
            snap = {"t": float(t)}
            for f in SNAPSHOT_FIELDS:
                if f"snapshots/{f}" in arrays:
                    snap[f] = arrays[f"snapshots/{f}"][i]
            if faces:
                snap["pressure_accel_faces"] = [np.asarray(c[i]) for c in faces]
            if coords:
                snap["grid_coords"] = [np.asarray(c[i]).copy() if (c.ndim >= 2 and c.shape[0] == len(times))
                                       else np.asarray(c).copy() for c in coords]
            snapshots.append(snap)
    debug = []
    if "debug/keys_json" in arrays:
        keys = _from_json_bytes(arrays["debug/keys_json"])
        count = len(arrays[f"debug/{keys[0]}"]) if keys else 0
        debug = [{k: arrays[f"debug/{k}"][i].item() for k in keys} for i in range(count)]
    return results, snapshots, debug


def load_checkpoint(path, *, solver, config_path=None, verify_code: bool = True) -> dict:
    """Validate a checkpoint and restore ``solver`` from it (checkpoint.py:
    190-225).  Returns time, step, state phase, dt candidate / effective,
    terminal clamp flag, grid hash, the state fields as the solver holds
    them, results, snapshots and debug history."""
    with np.load(path, allow_pickle=False) as data:
        arrays = {k: data[k] for k in data.files if k != "__manifest_json__"}
        manifest = _from_json_bytes(data["__manifest_json__"])
    _validate(manifest, arrays, solver, config_path, verify_code)
    st = _restore_state_dict(arrays)
    if st["geometric_phase"]:
        raise CheckpointError("checkpoint holds geometric phase state, which this package's step does not carry")
    fields = solver.restore_checkpoint_state(st)
    results, snapshots, debug = _restore_outputs(arrays)

    def opt(key):
        v = manifest.get(key)
        return None if v is None else float(v)
    out = {
        "t": float(manifest["time"]),
        "step": int(manifest["step"]),
        "state_phase": manifest.get("state_phase", "post_step"),
        "dt_candidate": opt("dt_candidate"),
        "dt_effective": opt("dt_effective"),
        "terminal_clamped": bool(manifest.get("terminal_clamped", False)),
        "grid_hash": manifest.get("grid_hash"),
        "results": results,
        "snapshots": snapshots,
        "debug_history": debug,
    }
    out.update(fields)
    return out
