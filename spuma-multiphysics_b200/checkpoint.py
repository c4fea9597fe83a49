"""Schema-3 ReactiveFoam checkpoints on the host: the binary conserved state and
thermodynamic seeds (`reactiveState.bin`), the identity dictionary
(`reactiveStateIdentity`), the sha256 manifest (`reactiveCheckpointComplete`)
and the atomic directory commit (src/reactiveFoam/reactiveCheckpoint.H:1-123,
the writer and reader the solver uses at src/reactiveFoam/ReactiveFoam.C:1099-1187
and :1316-1390).

`reactiveState.bin` is, little-endian and packed:

    u64 magic 0x524643484b505433, u64 endian 0x0102030405060708,
    u64 sizeof(double) = 8, u64 cells, u64 variables, u64 state bytes (176)
    u64 steps, u64 retries, f64 time, lastDt, velocityScale, energyScale
    f64 initial[variables], f64 boundary[variables]
    f64 q[cells][variables]                      (cell-major)
    ReactiveThermoState states[cells]            (176 bytes each)

A checkpoint is a time directory holding that file, the identity dictionary,
any other fields, and the manifest naming every regular file with its sha256.
A step driver restarts from the conserved state and the saved seeds exactly
(`Flow.save_checkpoint` / `Flow.load_checkpoint`).
"""
import ctypes as C
import hashlib
import itertools
import math
import os
import re
import shutil
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from ._abi import THERMO_DTYPE

MAGIC = 0x524643484B505433
ENDIAN = 0x0102030405060708
MARKER = "reactiveCheckpointComplete"
SIGNATURE = "ReactiveFoam checkpoint 3"
STATE_FILE = "reactiveState.bin"
IDENTITY_FILE = "reactiveStateIdentity"
_HEADER = struct.Struct("<6Q")
_HISTORY = struct.Struct("<2Q4d")


class CheckpointError(RuntimeError):
    pass


def _demand(ok, message):
    if not ok:
        raise CheckpointError(message)


@dataclass
class History:
    """Accepted-step history carried by a checkpoint (CheckpointHistory,
    reactiveCheckpoint.H:3-8): the conservation baseline and the accumulated
    boundary integral per variable, the counters, the physical time, the last
    step and the conservation scales."""
    initial: np.ndarray
    boundary: np.ndarray
    steps: int = 0
    retries: int = 0
    time: float = 0.0
    last_dt: float = 0.0
    velocity_scale: float = 1.0
    energy_scale: float = 0.0
    loaded: bool = field(default=False, compare=False)


def time_name(t, precision=6):
    """The time directory name of physical time t: OpenFOAM's default
    Time::timeName (general floating-point format, 6 significant digits)."""
    text = f"{t:.{precision}g}"
    return text


def identity_hash(text):
    """A 64-character lowercase hexadecimal digest (reactiveCheckpointIdentity.h:11-13)."""
    return isinstance(text, str) and len(text) == 64 and all(c in "0123456789abcdef" for c in text)


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for block in iter(lambda: f.read(1 << 22), b""):
            h.update(block)
    return h.hexdigest()


# ------------------------------------------------------------------ state file
def write_state(path, q, states, history):
    """Write `reactiveState.bin` (reactiveCheckpoint.H:35-48). q: (cells, nv)
    FP64; states: THERMO_DTYPE (cells,) or (cells, 176) bytes."""
    q = np.ascontiguousarray(q, dtype="<f8")
    _demand(q.ndim == 2, "q must be (cells, variables)")
    cells, nv = q.shape
    raw = np.ascontiguousarray(states).view(np.uint8).reshape(-1)
    _demand(raw.size == cells * THERMO_DTYPE.itemsize, "one 176-byte thermodynamic state per cell")
    initial = np.ascontiguousarray(history.initial, dtype="<f8")
    boundary = np.ascontiguousarray(history.boundary, dtype="<f8")
    _demand(initial.shape == (nv,) and boundary.shape == (nv,), "history integrals need one value per variable")
    with open(path, "wb") as out:
        out.write(_HEADER.pack(MAGIC, ENDIAN, 8, cells, nv, THERMO_DTYPE.itemsize))
        out.write(_HISTORY.pack(int(history.steps), int(history.retries), float(history.time),
                                float(history.last_dt), float(history.velocity_scale), float(history.energy_scale)))
        out.write(initial.tobytes())
        out.write(boundary.tobytes())
        out.write(q.tobytes())
        out.write(raw.tobytes())
        out.flush()
        os.fsync(out.fileno())


def read_state(path, cells=None, variables=None, time_dir=None):
    """Read and validate `reactiveState.bin` (reactiveCheckpoint.H:69-94):
    layout header, mesh size and variable count (when given), a finite history
    whose time names the directory (when `time_dir` is given), finite
    integrals, no trailing data. Returns (q (cells, nv), states THERMO_DTYPE,
    History)."""
    data = Path(path).read_bytes()
    _demand(len(data) >= _HEADER.size + _HISTORY.size, "Incomplete checkpoint state")
    magic, endian, scalar, n, nv, state_bytes = _HEADER.unpack_from(data, 0)
    _demand(magic == MAGIC and endian == ENDIAN and scalar == 8 and state_bytes == THERMO_DTYPE.itemsize
            and (cells is None or n == cells) and (variables is None or nv == variables),
            "Checkpoint layout/mesh/closure mismatch; explicit migration required")
    steps, retries, t, last_dt, vscale, escale = _HISTORY.unpack_from(data, _HEADER.size)
    _demand(math.isfinite(t) and (time_dir is None or time_name(t) == Path(time_dir).name)
            and math.isfinite(last_dt) and last_dt >= 0 and math.isfinite(vscale) and vscale > 0
            and math.isfinite(escale) and escale > 0, "Invalid checkpoint time/history")
    offset = _HEADER.size + _HISTORY.size
    need = offset + 2 * nv * 8 + n * nv * 8 + n * state_bytes
    _demand(len(data) >= need, "Incomplete checkpoint state")
    _demand(len(data) == need, "Checkpoint state has unexpected trailing data")
    initial = np.frombuffer(data, "<f8", nv, offset).copy()
    boundary = np.frombuffer(data, "<f8", nv, offset + nv * 8).copy()
    _demand(np.isfinite(initial).all(), "Invalid checkpoint conservation baseline")
    _demand(np.isfinite(boundary).all(), "Invalid checkpoint boundary integral")
    offset += 2 * nv * 8
    q = np.frombuffer(data, "<f8", n * nv, offset).reshape(n, nv).copy()
    _demand(np.isfinite(q).all(), "Checkpoint field/binary conserved state mismatch")
    offset += n * nv * 8
    states = np.frombuffer(data, THERMO_DTYPE, n, offset).copy()
    history = History(initial, boundary, steps, retries, t, last_dt, vscale, escale, loaded=True)
    return q, states, history


# ------------------------------------------------------------- identity file
def write_identity(path, fingerprint, physical_model_hash, numerical_policy_hash, species_count, closure,
                   location=None, restart_policy_hash=None):
    """The identity dictionary (ReactiveFoam.C:1376-1386) as an OpenFOAM ASCII
    dictionary; the hashes are quoted strings so a digest that starts with a
    digit is not read as a number."""
    for name, value in (("fingerprint", fingerprint), ("physicalModelHash", physical_model_hash),
                        ("numericalPolicyHash", numerical_policy_hash)):
        _demand(identity_hash(value), f"Invalid {name}")
    _demand(int(species_count) > 0 and closure and re.fullmatch(r"[A-Za-z0-9_.+-]+", closure) is not None,
            "Invalid species count or closure word")
    entries = [("fingerprint", f'"{fingerprint}"'), ("identitySchema", "3"),
               ("physicalModelHash", f'"{physical_model_hash}"'),
               ("numericalPolicyHash", f'"{numerical_policy_hash}"')]
    if restart_policy_hash is not None:
        _demand(identity_hash(restart_policy_hash), "Invalid restartNumericalPolicyHash")
        entries.append(("restartNumericalPolicyHash", f'"{restart_policy_hash}"'))
    entries += [("speciesCount", str(int(species_count))), ("closure", closure)]
    header = ["FoamFile", "{", "    version     2.0;", "    format      ascii;", "    class       dictionary;"]
    if location is not None:
        header.append(f'    location    "{location}";')
    header += [f"    object      {IDENTITY_FILE};", "}", ""]
    body = [key + " " * max(1, 20 - len(key)) + f"{value};" for key, value in entries]
    Path(path).write_text("\n".join(header + body) + "\n")


def read_identity(path):
    """Entries of an identity dictionary (the keys ReactiveFoam.C:1101-1107 reads)."""
    text = Path(path).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"FoamFile\s*\{[^}]*\}", "", text, flags=re.S)
    out = {}
    for key, value in re.findall(r"([A-Za-z_][A-Za-z0-9_]*)\s+([^;]*?)\s*;", text):
        value = value.strip()
        if value.startswith('"') and value.endswith('"'):
            value = value[1:-1]
        elif re.fullmatch(r"-?\d+", value):
            value = int(value)
        out[key] = value
    _demand("speciesCount" in out and "fingerprint" in out, "Invalid checkpoint identity")
    return out


# ------------------------------------------------------------- scalar fields
DIMENSIONS = {"p": "[1 -1 -2 0 0 0 0]", "T": "[0 0 0 1 0 0 0]", "rho": "[1 -3 0 0 0 0 0]"}


def write_field(path, name, values, dimensions, location=None):
    """A cell scalar field in OpenFOAM's binary volScalarField layout, internal
    values only (an empty boundaryField): the layout the reference's checkpoint
    tools read (tools/hem_checkpoint_batch.py:32-37)."""
    values = np.ascontiguousarray(values, dtype="<f8")
    head = ["FoamFile", "{", "    version     2.0;", "    format      binary;",
            '    arch        "LSB;label=32;scalar=64";', "    class       volScalarField;"]
    if location is not None:
        head.append(f'    location    "{location}";')
    head += [f"    object      {name};", "}", "", f"dimensions      {dimensions};", "",
             f"internalField   nonuniform List<scalar> {values.size}", "("]
    with open(path, "wb") as out:
        out.write(("\n".join(head)).encode())
        out.write(values.tobytes())
        out.write(b")\n;\n\nboundaryField\n{\n}\n")


def read_field(path, cells):
    """The internal values of a binary volScalarField of `cells` cells."""
    data = Path(path).read_bytes()
    m = re.search(rb"internalField\s+nonuniform\s+List<scalar>\s*(\d+)\s*\(", data)
    _demand(m is not None and int(m.group(1)) == cells, f"{path}: not a binary List<scalar> of {cells} values")
    _demand(len(data) >= m.end() + 8 * cells, f"{path}: truncated field")
    return np.frombuffer(data, "<f8", cells, m.end()).copy()


# ------------------------------------------------------------------ manifest
def _quote(name):
    # std::quoted: wrap in '"', escape '"' and '\\'
    return '"' + name.replace("\\", "\\\\").replace('"', '\\"') + '"'


def _manifest_entries(text):
    entries, i, n = [], 0, len(text)
    while True:
        while i < n and text[i].isspace():
            i += 1
        if i >= n:
            return entries
        j = i
        while j < n and not text[j].isspace():
            j += 1
        digest = text[i:j]
        i = j
        while i < n and text[i].isspace():
            i += 1
        _demand(i < n and text[i] == '"', "Invalid checkpoint manifest entry")
        i += 1
        name = []
        while i < n and text[i] != '"':
            if text[i] == "\\" and i + 1 < n:
                i += 1
            name.append(text[i])
            i += 1
        _demand(i < n, "Invalid checkpoint manifest entry")
        i += 1
        entries.append((digest, "".join(name)))


def verify(directory):
    """The complete marker and every file it names (reactiveCheckpoint.H:49-65):
    the signature line, well-formed digests and plain names, matching sha256,
    the state file and the identity present, more than two entries."""
    d = Path(directory)
    marker = d / MARKER
    _demand(marker.is_file(), "Incomplete checkpoint: missing/invalid complete marker")
    text = marker.read_text()
    first, _, rest = text.partition("\n")
    _demand(first == SIGNATURE, "Incomplete checkpoint: missing/invalid complete marker")
    state = identity = False
    entries = _manifest_entries(rest)
    for digest, name in entries:
        _demand(identity_hash(digest) and "/" not in name and name not in (".", "..", ""),
                "Invalid checkpoint manifest entry")
        _demand((d / name).is_file() and sha256(d / name) == digest, "Checkpoint checksum mismatch: " + name)
        state |= name == STATE_FILE
        identity |= name in (IDENTITY_FILE, IDENTITY_FILE + ".gz")
    _demand(state and identity and len(entries) > 2, "Incomplete checkpoint manifest")


def _fsync(path, directory=False):
    fd = os.open(path, os.O_RDONLY | (os.O_DIRECTORY if directory else 0))
    try:
        os.fsync(fd)
    finally:
        os.close(fd)


_RENAME_EXCHANGE = 2
_AT_FDCWD = -100


def _exchange(a, b):
    libc = C.CDLL(None, use_errno=True)
    fn = getattr(libc, "renameat2", None)
    if fn is None:
        raise CheckpointError("atomic directory exchange needs renameat2")
    fn.argtypes = [C.c_int, C.c_char_p, C.c_int, C.c_char_p, C.c_uint]
    if fn(_AT_FDCWD, os.fsencode(a), _AT_FDCWD, os.fsencode(b), _RENAME_EXCHANGE) != 0:
        raise CheckpointError(f"atomic directory exchange: {b}: {os.strerror(C.get_errno())}")


class Transaction:
    """Write a checkpoint into a hidden staging copy of the time directory and
    swap it in atomically (reactiveCheckpoint.H:95-122): the existing
    directory's files are carried over, the staged files are fsynced, the
    manifest names each with its sha256, and the staged directory replaces the
    target by rename (new) or renameat2 exchange (existing)."""
    _sequence = itertools.count(1)

    def __init__(self, root, time, run_id):
        self.root = Path(root)
        self.target = self.root / time
        self.stage = self.root / f".reactive-checkpoint-{run_id}-{next(Transaction._sequence)}"
        self.stage.mkdir()
        try:
            if self.target.exists():
                for entry in self.target.iterdir():
                    dst = self.stage / entry.name
                    if entry.is_dir() and not entry.is_symlink():
                        shutil.copytree(entry, dst, symlinks=True)
                    else:
                        shutil.copy2(entry, dst, follow_symlinks=False)
        except BaseException:
            shutil.rmtree(self.stage, ignore_errors=True)
            raise
        (self.stage / MARKER).unlink(missing_ok=True)

    def path(self):
        return self.stage

    def check_field(self, name):
        _demand(not (self.target / name).exists() or (self.target / name).is_file(),
                f"Failed to write checkpoint {name} is not a regular file")
        if (self.stage / name).is_symlink():
            (self.stage / name).unlink()

    def commit(self):
        files = sorted(p for p in self.stage.iterdir() if p.is_file() and not p.is_symlink())
        lines = [SIGNATURE]
        for f in files:
            _fsync(f)
            lines.append(f"{sha256(f)} {_quote(f.name)}")
        marker = self.stage / MARKER
        with open(marker, "w") as out:
            out.write("\n".join(lines) + "\n")
            out.flush()
            os.fsync(out.fileno())
        _fsync(self.stage, directory=True)
        if self.target.exists():
            _exchange(self.stage, self.target)
        else:
            os.rename(self.stage, self.target)
        _fsync(self.root, directory=True)

    def close(self):
        shutil.rmtree(self.stage, ignore_errors=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False


def save(root, q, states, history, identity, run_id="b200", extra=None, fields=("p", "T", "rho")):
    """Commit a checkpoint time directory named for history.time: the state
    file, the identity dictionary (`identity`: the keyword arguments of
    write_identity), the named state fields as binary cell fields and any
    `extra` files (name -> bytes). Returns the path."""
    time = time_name(history.time)
    with Transaction(root, time, run_id) as tx:
        for name in fields:
            tx.check_field(name)
            write_field(tx.path() / name, name, np.asarray(states[name]), DIMENSIONS[name], location=time)
        for name, payload in (extra or {}).items():
            tx.check_field(name)
            (tx.path() / name).write_bytes(payload)
        tx.check_field(IDENTITY_FILE)
        write_identity(tx.path() / IDENTITY_FILE, location=time, **identity)
        tx.check_field(STATE_FILE)
        write_state(tx.path() / STATE_FILE, q, states, history)
        tx.commit()
    return Path(root) / time


def load(directory, cells=None, variables=None):
    """Verify a committed checkpoint and read its state: (q, states, History,
    identity entries)."""
    verify(directory)
    q, states, history = read_state(Path(directory) / STATE_FILE, cells, variables, time_dir=directory)
    ident = None
    for name in (IDENTITY_FILE,):
        if (Path(directory) / name).is_file():
            ident = read_identity(Path(directory) / name)
    return q, states, history, ident


def flash_batch(directory, species=1, select="all"):
    """A flash batch from a checkpoint, as the reference's checkpoint batch
    tool forms one (tools/hem_checkpoint_batch.py:82-99) without the capillary
    terms: per selected cell its total density, internal energy density
    (rho E - |rho u|^2 / 2 rho, the flash input) and the committed state as the
    seed. select: "all", "liquid" (cells holding liquid) or "gas"."""
    q, states, _ = read_state(Path(directory) / STATE_FILE)
    rho = q[:, :species].sum(axis=1)
    internal = q[:, species + 3] - .5 * (q[:, species:species + 3] ** 2).sum(axis=1) / rho
    liquid = states["liquidMass"][:, 0] > 0
    mask = {"all": np.ones(len(q), bool), "liquid": liquid, "gas": ~liquid}[select]
    index = np.flatnonzero(mask)
    return rho[index], internal[index], states[index], index
