"""Exact-resume side-car: the part of a DEM run's state that the .bin
format does not hold.

A run restarted from a .bin alone is not the continuous run: the file has no
contact history (``contacts``, ``distmod``, ``delta_t``), no previous
accelerations (``acc``, ``angacc`` and the walls' ``acc``) that the
three-term Taylor integrator uses, and the loop counter starts again at 0,
which zeroes those accelerations (src/integration.cuh:74-81, ``iter`` local
to DEM::startTime, src/device.cu:926).  This module writes those arrays to a
side-car file next to the unchanged .bin and loads them into a reopened
engine, so that the resumed run continues bit for bit.

Side-car layout (little endian): the 12-byte magic, then uint32 version, np,
contact capacity, nw; then, in the order of ``FIELDS``, each field as a
uint64 byte count followed by the bytes of ``Engine.get(field)``.
"""
from __future__ import annotations

import os
import struct

import numpy

from .engine import Engine

MAGIC = b"SPHB-RESUME\x00"
VERSION = 1
FIELDS = ("contacts", "distmod", "delta_t", "acc", "angacc", "walls_acc", "iter",
          "velocity_state")


class ResumeError(ValueError):
    pass


def side_car_path(bin_path) -> str:
    return os.fspath(bin_path) + ".resume"


def write_resume(engine: Engine, path) -> None:
    """Writes the engine's side-car state to ``path``."""
    info = engine.info()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<4I", VERSION, info.np, info.capacity, info.nw))
        for name in FIELDS:
            a = numpy.ascontiguousarray(engine.get(name))
            f.write(struct.pack("<Q", a.nbytes))
            f.write(a.tobytes())


def read_resume(path) -> dict:
    """Reads a side-car file: a dict with 'np', 'capacity', 'nw' and the raw
    bytes of every field."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:len(MAGIC)] != MAGIC:
        raise ResumeError(f"{path}: not a resume side-car")
    pos = len(MAGIC)
    version, np_, cap, nw = struct.unpack_from("<4I", buf, pos)
    pos += 16
    if version != VERSION:
        raise ResumeError(f"{path}: side-car version {version}, expected {VERSION}")
    out = {"np": np_, "capacity": cap, "nw": nw}
    for name in FIELDS:
        if pos + 8 > len(buf):
            raise ResumeError(f"{path}: truncated before {name}")
        (n,) = struct.unpack_from("<Q", buf, pos)
        pos += 8
        if pos + n > len(buf):
            raise ResumeError(f"{path}: truncated in {name}")
        out[name] = buf[pos:pos + n]
        pos += n
    if pos != len(buf):
        raise ResumeError(f"{path}: {len(buf) - pos} trailing bytes")
    return out


def apply_resume(engine: Engine, state: dict) -> None:
    """Loads side-car state into an engine opened from the matching .bin."""
    info = engine.info()
    if (state["np"], state["capacity"], state["nw"]) != (info.np, info.capacity, info.nw):
        raise ResumeError(
            f"side-car for np={state['np']}, capacity={state['capacity']}, nw={state['nw']} "
            f"does not match the engine (np={info.np}, capacity={info.capacity}, nw={info.nw})")
    for name in FIELDS:
        dtype = numpy.uint32 if name == "contacts" else (
            numpy.int64 if name in ("iter", "velocity_state") else numpy.float64)
        arr = numpy.frombuffer(state[name], dtype=dtype)
        if arr.nbytes != engine.field_bytes(name):
            raise ResumeError(f"side-car field {name} has {arr.nbytes} bytes, "
                              f"the engine expects {engine.field_bytes(name)}")
        engine.set(name, arr)


def write_bin_with_resume(engine: Engine, bin_path) -> str:
    """Writes the .bin (unchanged format) and its side-car; returns the
    side-car's path."""
    engine.write_bin(bin_path)
    sc = side_car_path(bin_path)
    write_resume(engine, sc)
    return sc


def open_resumed(bin_path, **engine_kwargs) -> Engine:
    """Opens an engine from a .bin and, when its side-car exists, loads it."""
    e = Engine(os.fspath(bin_path), **engine_kwargs)
    sc = side_car_path(bin_path)
    if os.path.exists(sc):
        try:
            apply_resume(e, read_resume(sc))
        except Exception:
            e.close()
            raise
    return e
