"""The saved-model format (gprx's format_version 1: config.json and
model.safetensors, docs/persist-format.md of the reference) read and written
on the host: round trips, the file layout a reader without gprx relies on
(column-major tensors, 8-byte aligned data, plain JSON), the kernel tree's
JSON (left-nested binary sum / product, flattened on read), and the
refusals of files this backend does not read.
"""

import ctypes as C
import json
import math
import os
import struct

import numpy as np
import pytest

import gprx_b200 as gx
from gprx_b200 import _lib as L


def nodes_arr(nodes):
    arr = (L.KernelNode * len(nodes))()
    for i, (k, a) in enumerate(nodes):
        arr[i].kind, arr[i].arg = k, a
    return arr


def write(dirname, n=7, d=3, nodes=((1, 3), (10, 0), (2, 2), (12, 0), (11, 3), (13, 0)), factor=None, ids=None,
          jitter=None, seed=0):
    rs = np.random.RandomState(seed)
    x = rs.standard_normal(n * d)
    y = rs.standard_normal(n)
    nodes = list(nodes)
    n_params = gx.KernelSpec.from_nodes(nodes, [0.0] * 64).num_params()
    theta = np.log(rs.uniform(0.2, 3.0, size=n_params + 1))
    o = L.Options()
    L.lib().gprx_options_default(C.byref(o))
    if jitter:
        o.jitter_kind, o.jitter_initial, o.jitter_multiplier, o.jitter_max_retries, o.jitter_max = jitter
    l = a = None
    kind = 0
    if factor is not None:
        l, a, kind = factor
    idp = None
    if ids is not None:
        ids = np.asarray(ids, dtype=np.uint64)
        idp = ids.ctypes.data_as(L.U64)
    st = L.lib().gprx_persist_write(str(dirname).encode(), L.ptr(x), n, d, L.ptr(y), nodes_arr(nodes), len(nodes),
                                    L.ptr(theta), theta.size, C.byref(o), L.ptr(l) if l is not None else None,
                                    L.ptr(a) if a is not None else None, kind, 0.0, idp, 11)
    assert st == 0, L.last_error().message
    return x, y, theta, nodes


def read(dirname):
    info = gx.LoadedGpr.inspect(dirname)
    nodes = (L.KernelNode * info.n_nodes)()
    theta = np.zeros(info.n_theta)
    x = np.zeros(info.n * info.d)
    y = np.zeros(info.n)
    l = np.zeros(info.n * info.n) if info.has_factor else None
    a = np.zeros(info.n) if info.has_factor else None
    ids = np.zeros(info.n, dtype=np.uint64) if info.factor_kind == 1 else None
    gx.api.check(L.lib().gprx_persist_read(str(dirname).encode(), nodes, L.ptr(theta), L.ptr(x), L.ptr(y),
                                           L.ptr(l) if l is not None else None, L.ptr(a) if a is not None else None,
                                           ids.ctypes.data_as(L.U64) if ids is not None else None))
    return info, [(nd.kind, nd.arg) for nd in nodes], theta, x, y, l, a, ids


def load_tensors(path):
    """A reader without gprx (NumPy only): header length, JSON header, bytes."""
    raw = open(path, "rb").read()
    (hl,) = struct.unpack("<Q", raw[:8])
    header = json.loads(raw[8:8 + hl])
    body = 8 + hl
    out = {}
    for name, meta in header.items():
        lo, hi = meta["data_offsets"]
        assert meta["dtype"] == "F64" and (body + lo) % 8 == 0
        out[name] = np.frombuffer(raw[body + lo:body + hi], dtype="<f8").reshape(meta["shape"], order="F")
    return out


def test_round_trip_without_factor(tmp_path):
    x, y, theta, nodes = write(tmp_path / "m", jitter=(1, 1e-8, 10.0, 5, 1e-3))
    info, n2, th2, x2, y2, l2, a2, _ = read(tmp_path / "m")
    assert (info.n, info.d, info.has_factor, info.factor_kind) == (7, 3, 0, 0)
    assert n2 == nodes
    assert np.array_equal(x2, x) and np.array_equal(y2, y)
    assert np.all(np.abs(th2 - theta) <= 4e-16 * np.maximum(1, np.abs(theta)))  # stored as values, read as logs
    j = info.jitter
    assert (j.jitter_kind, j.jitter_initial, j.jitter_multiplier, j.jitter_max_retries, j.jitter_max) == \
        (1, 1e-8, 10.0, 5, 1e-3)


def test_files_are_readable_without_gprx(tmp_path):
    n, d = 9, 2
    rs = np.random.RandomState(3)
    lmat = np.tril(rs.standard_normal((n, n))) + 3 * np.eye(n)
    lmat_with_upper = lmat + np.triu(np.ones((n, n)), 1)  # the writer must zero the upper part
    alpha = rs.standard_normal(n)
    x, y, theta, nodes = write(tmp_path / "m", n=n, d=d, nodes=((11, 2),),
                               factor=(lmat_with_upper.reshape(-1, order="F").copy(), alpha, 0))
    cfg = json.load(open(tmp_path / "m" / "config.json"))
    assert cfg["format_version"] == 1 and cfg["n"] == n and cfg["d"] == d
    assert cfg["has_factor"] is True and cfg["factor_kind"] == "llt"
    assert cfg["x_transform"] == "identity" and cfg["y_transform"] == "identity"
    ls = cfg["kernel"]["rbf_ard"]["lengthscales"]
    assert [v["value"] for v in ls] == [math.exp(t) for t in theta[:2]]
    assert cfg["likelihood"]["noise_variance"]["value"] == math.exp(theta[-1])
    t = load_tensors(tmp_path / "m" / "model.safetensors")
    assert t["x"].shape == (n, d) and np.array_equal(t["x"], x.reshape(n, d, order="F"))
    assert np.array_equal(t["y"], y) and np.array_equal(t["alpha"], alpha)
    assert np.array_equal(t["l"], lmat)  # column-major, zero above the diagonal
    info, _, _, _, _, l2, a2, _ = read(tmp_path / "m")
    assert np.array_equal(l2.reshape(n, n, order="F"), lmat) and np.array_equal(a2, alpha)


def test_kernel_json_nests_and_flattens(tmp_path):
    nodes = ((2, 3), (12, 0), (1, 2), (10, 0), (13, 0), (11, 3))  # Const × (Rbf + Periodic) × RbfArd(3)
    write(tmp_path / "m", nodes=nodes)
    k = json.load(open(tmp_path / "m" / "config.json"))["kernel"]
    # three factors: product(product(constant, sum(rbf, periodic)), rbf_ard)
    outer = k["product"]
    assert "rbf_ard" in outer["right"] and "constant" in outer["left"]["product"]["left"]
    assert set(outer["left"]["product"]["right"]["sum"]) == {"left", "right"}
    _, n2, _, _, _, _, _, _ = read(tmp_path / "m")
    assert n2 == list(nodes)


def test_online_ids_round_trip(tmp_path):
    n = 5
    l = np.tril(np.ones((n, n))).reshape(-1, order="F").copy()
    write(tmp_path / "m", n=n, d=1, nodes=((10, 0),), factor=(l, np.ones(n), 1), ids=[0, 2, 3, 7, 9])
    info, _, _, _, _, _, _, ids = read(tmp_path / "m")
    assert info.factor_kind == 1 and info.next_point_id == 11 and list(ids) == [0, 2, 3, 7, 9]
    cfg = json.load(open(tmp_path / "m" / "config.json"))
    assert cfg["point_ids"] == [0, 2, 3, 7, 9] and cfg["next_point_id"] == 11


def test_hand_written_config_in_the_documented_form(tmp_path):
    # a Constant × RBF model with identity maps, written by hand from the format's schema
    d = tmp_path / "m"
    os.makedirs(d)
    cfg = {
        "format_version": 1, "n": 2, "d": 1, "has_factor": False, "factor_kind": "llt",
        "kernel": {"product": {
            "left": {"constant": {"constant": {"value": 1.5, "lo": 1e-5, "hi": 1e5}}},
            "right": {"rbf": {"lengthscale": {"value": 0.75, "lo": 1e-5, "hi": 1e5}}}}},
        "likelihood": {"noise_variance": {"value": 0.1, "lo": 1e-5, "hi": 1e5}},
        "jitter": {"fixed": {"jitter": 0.0}}, "distance_cache": "always",
        "x_unfitted": "identity", "y_unfitted": "identity", "x_transform": "identity", "y_transform": "identity",
        "an_unknown_key": [1, 2, 3],
    }
    json.dump(cfg, open(d / "config.json", "w"), indent=2)
    header = json.dumps({"x": {"dtype": "F64", "shape": [2, 1], "data_offsets": [0, 16]},
                         "y": {"dtype": "F64", "shape": [2], "data_offsets": [16, 32]}})
    header += " " * ((8 - (8 + len(header)) % 8) % 8)
    with open(d / "model.safetensors", "wb") as fh:
        fh.write(struct.pack("<Q", len(header)) + header.encode() + np.array([0.0, 1.0, 0.5, -0.5]).tobytes())
    info, nodes, theta, x, y, _, _, _ = read(d)
    assert nodes == [(2, 2), (12, 0), (10, 0)]
    assert np.allclose(np.exp(theta), [1.5, 0.75, 0.1], rtol=1e-15)
    assert list(x) == [0.0, 1.0] and list(y) == [0.5, -0.5]


@pytest.mark.parametrize("edit,err", [
    (lambda c: c.update(format_version=2), gx.UnsupportedPersistVersion),
    (lambda c: c.update(x_transform="standardize"), gx.PersistFailed),
    (lambda c: c.update(kernel={"matern": {"lengthscale": {"value": 1.0, "lo": 1e-5, "hi": 1e5}, "nu": "half"}}),
     gx.PersistFailed),
    (lambda c: c.update(model="sgpr"), gx.PersistFailed),
    (lambda c: c.update(precision="single"), gx.PersistFailed),
    (lambda c: c["likelihood"]["noise_variance"].update(value=2e5), gx.PersistFailed),
], ids=["version", "transform", "kernel", "wrong-model", "precision", "bound"])
def test_refusals(tmp_path, edit, err):
    write(tmp_path / "m", n=4, d=1, nodes=((10, 0),))
    cfg = json.load(open(tmp_path / "m" / "config.json"))
    edit(cfg)
    json.dump(cfg, open(tmp_path / "m" / "config.json", "w"))
    with pytest.raises(err):
        gx.LoadedGpr.inspect(tmp_path / "m")


def test_bad_tensors_are_refused(tmp_path):
    write(tmp_path / "m", n=4, d=1, nodes=((10, 0),))
    path = tmp_path / "m" / "model.safetensors"
    raw = bytearray(open(path, "rb").read())
    (hl,) = struct.unpack("<Q", raw[:8])
    raw[8 + hl:8 + hl + 8] = struct.pack("<d", float("nan"))  # x[0]
    open(path, "wb").write(bytes(raw))
    with pytest.raises(gx.PersistFailed):
        gx.LoadedGpr.inspect(tmp_path / "m")
    os.remove(path)
    with pytest.raises(gx.PersistFailed):
        gx.LoadedGpr.inspect(tmp_path / "m")
