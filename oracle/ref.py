"""ctypes wrapper of oracle/_ref/libykref.so, the reference YKCBCT CUDA build
(oracle/ref_build.py, oracle/ref_driver.cu).  TEST INFRASTRUCTURE ONLY.

The reference aborts its process on a CUDA error, so every call runs in a
child process started with ``spawn``.  Inputs and outputs are numpy float32
arrays: projections [view][v][u], volumes [z][y][x].
"""
from __future__ import annotations

import ctypes as C
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libykref.so")


def available() -> bool:
    return os.path.exists(LIB)


def _load():
    lib = C.CDLL(LIB)
    lib.ykref_last_error.restype = C.c_char_p
    for name in ("ykref_fdk", "ykref_fdk_stages", "ykref_fdk_time", "ykref_joseph_fp",
                 "ykref_joseph_bp", "ykref_bp_pseudo", "ykref_siddon_fp", "ykref_siddon_bp",
                 "ykref_cgls"):
        getattr(lib, name).restype = C.c_int
    return lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _child(op, scan_kw, grid_kw, filt_kw, paths, out_dir, opts, q):
    # the reference library logs to stdout; keep the caller's stdout for its
    # own output (the benchmark's single JSON line)
    sys.stdout.flush()
    os.dup2(2, 1)
    try:
        from fdk_cuda_impl_b200.geometry import CircularScan, RampFilter, VolumeGrid
        arrays = [np.load(p) for p in paths]
        scan = CircularScan(**scan_kw)
        grid = VolumeGrid(**grid_kw)
        lib = _load()
        s = scan.spec()
        v = grid.struct()
        dev = C.c_int(opts.get("device", 0))
        nproj = (scan.total_views, scan.rows, scan.channels)
        if op == "fdk":
            f = RampFilter(**filt_kw).struct()
            proj = np.ascontiguousarray(arrays[0], dtype=np.float32)
            out = np.zeros(grid.shape, dtype=np.float32)
            rc = lib.ykref_fdk(C.byref(s), C.byref(v), C.byref(f), _fp(proj), _fp(out),
                               C.c_int(opts.get("batch_views", 0)), dev)
            res = out
        elif op == "fdk_stages":
            f = RampFilter(**filt_kw).struct()
            proj = np.ascontiguousarray(arrays[0], dtype=np.float32)
            out = np.zeros(grid.shape, dtype=np.float32)
            pw = np.zeros((32, scan.rows, scan.channels), dtype=np.float32)
            fl = np.zeros_like(pw)
            first, count = C.c_int(0), C.c_int(0)
            rc = lib.ykref_fdk_stages(C.byref(s), C.byref(v), C.byref(f), _fp(proj), _fp(out),
                                      _fp(pw), _fp(fl), C.byref(first), C.byref(count), dev)
            res = (out, pw[:count.value], fl[:count.value], first.value)
        elif op == "cgls":
            proj = np.ascontiguousarray(arrays[0], dtype=np.float32)
            out = np.zeros(grid.shape, dtype=np.float32)
            ms = C.c_float(0.0)
            rc = lib.ykref_cgls(C.byref(s), C.byref(v), _fp(proj), _fp(out),
                                C.c_int(opts["n_iter"]), C.c_int(opts.get("matched", 1)),
                                C.byref(ms), dev)
            res = (out, ms.value)
        elif op == "fdk_time":
            f = RampFilter(**filt_kw).struct()
            proj = np.ascontiguousarray(arrays[0], dtype=np.float32)
            ms = (C.c_float * 2)()
            out = np.zeros(grid.shape, dtype=np.float32)
            rc = lib.ykref_fdk_time(C.byref(s), C.byref(v), C.byref(f), _fp(proj),
                                    C.c_int(opts["warmup"]), C.c_int(opts["reps"]), ms, _fp(out),
                                    dev)
            res = (ms[0], ms[1], out)
        else:
            x = np.ascontiguousarray(arrays[0], dtype=np.float32)
            out = np.zeros(nproj if op in ("fp", "siddon_fp") else grid.shape, dtype=np.float32)
            ms = C.c_float(0.0)
            fn = {"fp": lib.ykref_joseph_fp, "bp": lib.ykref_joseph_bp,
                  "bp_pseudo": lib.ykref_bp_pseudo, "siddon_fp": lib.ykref_siddon_fp,
                  "siddon_bp": lib.ykref_siddon_bp}[op]
            rc = fn(C.byref(s), C.byref(v), _fp(x), _fp(out), C.c_int(opts.get("warmup", 0)),
                    C.c_int(opts.get("reps", 0)), C.byref(ms), dev)
            res = (out, ms.value)
        if rc != 0:
            q.put(("error", lib.ykref_last_error().decode()))
        else:
            q.put(("ok", _to_files(res, out_dir)))
    except Exception as e:  # reported to the parent
        q.put(("error", repr(e)))


def _to_files(res, out_dir):
    """Arrays of a result travel back as .npy files (they can be GBs)."""
    if isinstance(res, np.ndarray):
        path = os.path.join(out_dir, f"out{len(os.listdir(out_dir))}.npy")
        np.save(path, res)
        return ("npy", path)
    if isinstance(res, tuple):
        return tuple(_to_files(r, out_dir) for r in res)
    return res


def _from_files(res):
    if isinstance(res, tuple) and len(res) == 2 and res[0] == "npy":
        return np.load(res[1])
    if isinstance(res, tuple):
        return tuple(_from_files(r) for r in res)
    return res


def _run(op, scan, grid, filt, arrays, **opts):
    import dataclasses
    import shutil
    import tempfile
    # inputs travel to the child as .npy files (they can be GBs)
    tmp_root = os.path.join(HERE, "_ref", "tmp")
    os.makedirs(tmp_root, exist_ok=True)
    tmp = tempfile.mkdtemp(dir=tmp_root)
    try:
        paths = []
        for i, a in enumerate(arrays):
            paths.append(os.path.join(tmp, f"in{i}.npy"))
            np.save(paths[-1], np.ascontiguousarray(a, dtype=np.float32))
        ctx = mp.get_context("spawn")
        q = ctx.Queue()
        filt_kw = dataclasses.asdict(filt) if filt is not None else None
        out_dir = os.path.join(tmp, "out")
        os.makedirs(out_dir)
        p = ctx.Process(target=_child, args=(op, dataclasses.asdict(scan), dataclasses.asdict(grid),
                                             filt_kw, paths, out_dir, opts, q))
        p.start()
        try:
            status, res = q.get(timeout=opts.get("timeout", 900))
        finally:
            p.join(timeout=60)
        if status == "ok":
            res = _from_files(res)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    if status != "ok":
        raise RuntimeError(f"reference {op} failed: {res} (exit code {p.exitcode})")
    return res


def fdk(scan, grid, filt, proj, batch_views=0):
    """Reference FdkPipeline FDK of host projections -> volume."""
    return _run("fdk", scan, grid, filt, [proj], batch_views=batch_views)


def fdk_stages(scan, grid, filt, proj):
    """Reference FDK plus its last chunk's stage buffers:
    (volume, preweighted rows, filtered rows, first view of that chunk)."""
    return _run("fdk_stages", scan, grid, filt, [proj])


def fdk_time(scan, grid, filt, proj, warmup=2, reps=5, timeout=900):
    """(device-resident ms, host-input ms, volume) per full FDK sequence: host
    projections and volume in pinned memory; the volume is the last
    device-resident run's."""
    return _run("fdk_time", scan, grid, filt, [proj], warmup=warmup, reps=reps, timeout=timeout)


def cgls(scan, grid, proj, n_iter, matched=True, timeout=900):
    """Reference CglsAstraBackend from a zero volume with FP_Joseph and
    BP_Joseph (matched) or BP_FDK_PseudoMatched: (volume, run() ms)."""
    return _run("cgls", scan, grid, None, [proj], n_iter=n_iter, matched=int(matched),
                timeout=timeout)


def joseph_fp(scan, grid, volume, warmup=0, reps=0):
    """Reference FP_Joseph: (projections, ms per call when reps > 0)."""
    return _run("fp", scan, grid, None, [volume], warmup=warmup, reps=reps)


def siddon_fp(scan, grid, volume, warmup=0, reps=0):
    """Reference FP_Siddon: (projections, ms per call when reps > 0)."""
    return _run("siddon_fp", scan, grid, None, [volume], warmup=warmup, reps=reps)


def siddon_bp(scan, grid, proj, warmup=0, reps=0):
    """Reference BP_Siddon_RayDriven (clear volume): (volume, ms per call when reps > 0)."""
    return _run("siddon_bp", scan, grid, None, [proj], warmup=warmup, reps=reps)


def bp_pseudo(scan, grid, proj, warmup=0, reps=0):
    """Reference BP_FDK_PseudoMatched (clear volume): (volume, ms per call when reps > 0)."""
    return _run("bp_pseudo", scan, grid, None, [proj], warmup=warmup, reps=reps)


def joseph_bp(scan, grid, proj, warmup=0, reps=0):
    """Reference BP_Joseph (clear volume): (volume, ms per call when reps > 0)."""
    return _run("bp", scan, grid, None, [proj], warmup=warmup, reps=reps)
