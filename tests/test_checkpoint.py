"""CPU: schema-3 checkpoints (src/reactiveFoam/reactiveCheckpoint.H:1-123): the
state file's byte layout (read back by the reference's own checkpoint tool when
the reference tree is present), the manifest checks, the atomic commit over an
existing time directory, the reader's validation, and the identity dictionary."""
import importlib.util
import os
import struct
from pathlib import Path

import numpy as np
import pytest

from spuma_multiphysics_b200 import _abi as A, checkpoint as ck

HASH = "0123456789abcdef" * 4
IDENTITY = dict(fingerprint=HASH, physical_model_hash="f" * 64, numerical_policy_hash="a" * 64, species_count=4,
                closure="HEM")


def sample(cells=13, nv=5, seed=0, time=1e-7):
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(cells, nv))
    states = np.zeros(cells, dtype=A.THERMO_DTYPE)
    raw = states.view(np.uint8).reshape(cells, -1)
    raw[:] = rng.integers(0, 256, raw.shape, dtype=np.uint8)
    states["p"] = rng.uniform(1e5, 5e6, cells)
    states["T"] = rng.uniform(200, 320, cells)
    hist = ck.History(initial=rng.normal(size=nv), boundary=rng.normal(size=nv), steps=7, retries=2, time=time,
                      last_dt=1e-8, velocity_scale=412.5, energy_scale=3.5e9)
    return q, states, hist


def test_state_file_layout_and_round_trip(tmp_path):
    q, states, hist = sample()
    path = tmp_path / "reactiveState.bin"
    ck.write_state(path, q, states, hist)
    data = path.read_bytes()
    assert struct.unpack_from("<6Q", data) == (0x524643484B505433, 0x0102030405060708, 8, 13, 5, 176)
    assert struct.unpack_from("<2Q4d", data, 48) == (7, 2, 1e-7, 1e-8, 412.5, 3.5e9)
    assert len(data) == 48 + 48 + 2 * 5 * 8 + 13 * 5 * 8 + 13 * 176
    q2, s2, h2 = ck.read_state(path, 13, 5)
    assert np.array_equal(q2, q) and s2.tobytes() == states.tobytes()
    assert np.array_equal(h2.initial, hist.initial) and np.array_equal(h2.boundary, hist.boundary)
    assert (h2.steps, h2.retries, h2.time, h2.last_dt, h2.velocity_scale, h2.energy_scale) == (7, 2, 1e-7, 1e-8,
                                                                                              412.5, 3.5e9)


def test_reference_tool_reads_the_state_file(tmp_path):
    from oracle import oracle
    tool = oracle.REFERENCE / "tools" / "hem_checkpoint_batch.py"
    if not tool.is_file():
        pytest.skip("reference tree not present")
    spec = importlib.util.spec_from_file_location("hem_checkpoint_batch", tool)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    q, states, hist = sample(cells=29, nv=8, seed=3)
    ck.write_state(tmp_path / "reactiveState.bin", q, states, hist)
    rq, rstates = mod.read_state(tmp_path / "reactiveState.bin")
    assert np.array_equal(rq, q)
    assert rstates.tobytes() == states.tobytes()
    ck.write_field(tmp_path / "p", "p", states["p"], ck.DIMENSIONS["p"])
    assert np.array_equal(mod.read_field(tmp_path / "p", 29), states["p"])


def test_reader_validation(tmp_path):
    q, states, hist = sample()
    path = tmp_path / "s.bin"
    ck.write_state(path, q, states, hist)
    with pytest.raises(ck.CheckpointError, match="mismatch"):
        ck.read_state(path, cells=12)
    with pytest.raises(ck.CheckpointError, match="mismatch"):
        ck.read_state(path, variables=6)
    with pytest.raises(ck.CheckpointError, match="time/history"):
        ck.read_state(path, time_dir=tmp_path / "2e-07")
    assert ck.read_state(path, time_dir=tmp_path / "1e-07")[2].loaded
    path.write_bytes(path.read_bytes() + b"\0")
    with pytest.raises(ck.CheckpointError, match="trailing"):
        ck.read_state(path)
    bad = ck.History(**{**hist.__dict__, "energy_scale": 0.0})
    ck.write_state(path, q, states, bad)
    with pytest.raises(ck.CheckpointError, match="time/history"):
        ck.read_state(path)
    q[3, 2] = np.nan
    ck.write_state(path, q, states, hist)
    with pytest.raises(ck.CheckpointError, match="conserved"):
        ck.read_state(path)


def test_time_names():
    # OpenFOAM's default timeName: general format, 6 significant digits
    assert [ck.time_name(t) for t in (1e-8, 1e-4, 5e-5, 0.000123456789, 2.0, 0.1, 1e-07)] == [
        "1e-08", "0.0001", "5e-05", "0.000123457", "2", "0.1", "1e-07"]


def test_save_verify_load_and_atomic_replace(tmp_path):
    q, states, hist = sample()
    out = ck.save(tmp_path, q, states, hist, IDENTITY, extra={"U": b"field bytes"})
    assert out == tmp_path / "1e-07"
    lines = (out / ck.MARKER).read_text().splitlines()
    assert lines[0] == "ReactiveFoam checkpoint 3"
    assert [ln.split(" ", 1)[1] for ln in lines[1:]] == ['"T"', '"U"', '"p"', '"reactiveState.bin"',
                                                         '"reactiveStateIdentity"', '"rho"']
    for name in ("p", "T", "rho"):
        assert np.array_equal(ck.read_field(out / name, 13), states[name])
    ck.verify(out)
    q2, s2, h2, ident = ck.load(out, 13, 5)
    assert np.array_equal(q2, q) and s2.tobytes() == states.tobytes() and h2.steps == 7
    assert ident["fingerprint"] == HASH and ident["speciesCount"] == 4 and ident["identitySchema"] == 3
    assert ident["closure"] == "HEM"
    # an auxiliary file of the existing directory survives a new commit
    (out / "aux").write_bytes(b"kept")
    q3 = q * 2
    ck.save(tmp_path, q3, states, hist, IDENTITY)
    ck.verify(out)
    assert (out / "aux").read_bytes() == b"kept"
    assert np.array_equal(ck.load(out)[0], q3)
    assert not [p for p in tmp_path.iterdir() if p.name.startswith(".reactive-checkpoint")]


def test_manifest_rejections(tmp_path):
    q, states, hist = sample()
    out = ck.save(tmp_path, q, states, hist, IDENTITY, extra={"U": b"u"})
    # a changed byte
    raw = bytearray((out / "reactiveState.bin").read_bytes())
    raw[100] ^= 1
    (out / "reactiveState.bin").write_bytes(bytes(raw))
    with pytest.raises(ck.CheckpointError, match="checksum"):
        ck.verify(out)
    out = ck.save(tmp_path, q, states, hist, IDENTITY, extra={"U": b"u"})
    marker = (out / ck.MARKER).read_text()
    (out / ck.MARKER).write_text(marker.replace("checkpoint 3", "checkpoint 2"))
    with pytest.raises(ck.CheckpointError, match="marker"):
        ck.verify(out)
    lines = marker.splitlines()
    (out / ck.MARKER).write_text("\n".join(ln for ln in lines if "Identity" not in ln) + "\n")
    with pytest.raises(ck.CheckpointError, match="manifest"):
        ck.verify(out)
    (out / ck.MARKER).write_text(marker + f'{HASH} "../escape"\n')
    with pytest.raises(ck.CheckpointError, match="entry"):
        ck.verify(out)
    (out / ck.MARKER).write_text(marker + 'ABC "U"\n')
    with pytest.raises(ck.CheckpointError, match="entry"):
        ck.verify(out)
    (out / ck.MARKER).unlink()
    with pytest.raises(ck.CheckpointError, match="marker"):
        ck.verify(out)
    # the state file and the identity alone are not a complete checkpoint
    (tmp_path / "bare").mkdir()
    bare = ck.save(tmp_path / "bare", q, states, hist, IDENTITY, fields=())
    with pytest.raises(ck.CheckpointError, match="manifest"):
        ck.verify(bare)


def test_identity_dictionary(tmp_path):
    path = tmp_path / "reactiveStateIdentity"
    ck.write_identity(path, location="0.0001", restart_policy_hash="b" * 64, **IDENTITY)
    text = path.read_text()
    assert "FoamFile" in text and 'fingerprint         "0123' in text
    got = ck.read_identity(path)
    assert got["physicalModelHash"] == "f" * 64 and got["restartNumericalPolicyHash"] == "b" * 64
    with pytest.raises(ck.CheckpointError):
        ck.write_identity(path, **{**IDENTITY, "fingerprint": "XYZ"})


def test_flash_batch_selection(tmp_path):
    q, states, hist = sample(cells=10, nv=5)
    q[:, 0] = np.abs(q[:, 0]) + 1
    states["liquidMass"][:, 0] = 0
    states["liquidMass"][[2, 5], 0] = 1.5
    ck.write_state(tmp_path / ck.STATE_FILE, q, states, hist)
    rho, e, seeds, index = ck.flash_batch(tmp_path, select="liquid")
    assert list(index) == [2, 5]
    assert np.allclose(e, q[index, 4] - .5 * (q[index, 1:4] ** 2).sum(1) / q[index, 0])
    assert seeds.tobytes() == states[index].tobytes()
