"""Field evaluation inside application kernels (include/psr_field.cuh), the counterpart of
warp-psr's ``evaluate_field(field, point)`` on a ``device_field()`` handle
(src/warp_psr/device_field.py:91-142; the reference's tests/test_device_field.py).

A user kernel, compiled by nvcc with its default flags (FMA contraction on), evaluates the
handle of a reconstruction and must return bit for bit what ``result.evaluate`` returns,
inside, on and outside the cube and at non-finite points.  A handle built by hand without
the hash table (binary search of the keys, as the reference's find_key) must agree too, and
the reference's small adaptive field, evaluated the direct way and the cumulative way, must
match a scalar restatement of field.py:36-81,365-421 in the same precision."""
import ctypes
from pathlib import Path

import numpy as np
import pytest
import torch

from warp_psr_b200 import _lib, clouds, reconstruct
from warp_psr_b200.build import build_user_library

pytestmark = pytest.mark.gpu

KERNEL = Path(__file__).resolve().parent / "kernels" / "device_field_user.cu"


@pytest.fixture(scope="module")
def user_lib(tmp_path_factory):
    out = build_user_library([KERNEL], tmp_path_factory.mktemp("user") / "libdevice_field_user.so")
    lib = ctypes.CDLL(str(out))
    vp = ctypes.c_void_p
    lib.user_evaluate.argtypes = [ctypes.POINTER(_lib.FieldHandle), vp, ctypes.c_int64, vp, vp, vp, vp]
    lib.user_evaluate.restype = ctypes.c_int
    return lib


def user_query(lib, handle, q):
    dtype = torch.float64 if handle.dtype == _lib.PSR_FLOAT64 else torch.float32
    q = q.to(dtype).contiguous()
    n = q.shape[0]
    values = torch.empty(n, dtype=dtype, device="cuda")
    gradients = torch.empty((n, 3), dtype=dtype, device="cuda")
    valid = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.user_evaluate(ctypes.byref(handle), q.data_ptr(), n, values.data_ptr(), gradients.data_ptr(),
                             valid.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    return values, gradients, valid


def assert_same(actual, expected):
    for a, e in zip(actual, expected):
        np.testing.assert_array_equal(a.cpu().numpy(), e.cpu().numpy())


def queries(p, dtype):
    rng = np.random.default_rng(2026)
    lo, hi = p.min(0), p.max(0)
    inside = lo + (hi - lo) * rng.uniform(-0.15, 1.15, size=(4000, 3))
    special = np.array([[np.nan, 0, 0], [np.inf, 0, 0], [-np.inf, 0, 0], [0, 0, 0], [1e30, 0, 0]])
    return torch.tensor(np.concatenate([inside, p[:500], lo[None], hi[None], special]), dtype=dtype, device="cuda")


@pytest.mark.parametrize("dtype,precision", [(torch.float32, "input"), (torch.float64, "input"),
                                             (torch.float32, "mixed")])
def test_user_kernel_matches_result_evaluate(user_lib, dtype, precision):
    p, n = clouds.torus(20_000)
    result = reconstruct(torch.tensor(p, dtype=dtype, device="cuda"), torch.tensor(n, dtype=dtype, device="cuda"),
                         depth=6, full_depth=3, point_weight=2.0, precision=precision)
    field = result.device_field()
    handle = field.handle
    assert handle.keys == result.field.keys.data_ptr()
    assert handle.coefficients == result.field.coefficients.data_ptr()
    assert handle.cumulative == result.field.cumulative.data_ptr()
    assert handle.hash_slots and handle.count == result.field.keys.numel()
    assert handle.iso_value == result.iso_value
    q = queries(p, result.field.coefficients.dtype)
    actual = user_query(user_lib, handle, q)
    expected = result.evaluate(q)
    assert_same(actual, expected)
    valid = actual[2].cpu().numpy()
    assert valid[:-5].any() and not valid[-5:-2].any()
    assert np.isnan(actual[0].cpu().numpy()[valid == 0]).all()
    # a handle built without the table binary-searches the sorted keys: same bits
    bare = _lib.FieldHandle.from_buffer_copy(handle)
    bare.hash_slots = None
    bare.hash_mask = 0
    assert_same(user_query(user_lib, bare, q), expected)
    empty = user_query(user_lib, handle, q[:0])
    assert empty[0].numel() == 0


# ---------------------------------------------------------------- the reference's adaptive field
def adaptive_keys():
    keys = []
    for depth in range(3):
        for x in range((1 << depth) + 1):
            for y in range((1 << depth) + 1):
                for z in range((1 << depth) + 1):
                    if depth < 2 or (x <= 2 and y <= 2 and z <= 2):
                        keys.append((depth << 48) | (x << 32) | (y << 16) | z)
    return np.array(keys, np.int64)


def cumulative_of(keys, coeff, T):
    """field.py:187-203 in precision T: cumulative = coefficients + trilinear parent sum."""
    index = {int(k): i for i, k in enumerate(keys)}
    cum = coeff.astype(T).copy()
    for i, k in enumerate(keys):
        d, c = int(k) >> 48, [(int(k) >> s) & 65535 for s in (32, 16, 0)]
        if d == 0:
            continue
        value = T(0)
        for corner in range(8):
            par = [c[0] // 2 + corner // 4, c[1] // 2 + (corner // 2) % 2, c[2] // 2 + corner % 2]
            hw = T(1)
            for a in range(3):
                f = T(1) - abs(T(c[a]) * T(.5) - T(par[a]))
                hw = f if a == 0 else hw * f
            if hw > T(0):
                j = index.get(((d - 1) << 48) | (par[0] << 32) | (par[1] << 16) | par[2], -1)
                if j >= 0:
                    value = value + cum[j] * hw
        cum[i] = value + T(coeff[i])
    return cum


def restated_query(keys, coeff, cum, depth, L, tr, q, T):
    """One query by field.py:36-81 (cum None: direct) or :365-421 (cumulative), scalar T ops."""
    index = {int(k): i for i, k in enumerate(keys)}

    def find(d, x, y, z):
        return index.get((d << 48) | (x << 32) | (y << 16) | z, -1)

    L = [T(v) for v in L]
    tr = [T(v) for v in tr]
    q = [T(v) for v in q]
    with np.errstate(invalid="ignore", over="ignore"):
        p = [((L[3 * r] * q[0] + L[3 * r + 1] * q[1]) + L[3 * r + 2] * q[2]) + tr[r] for r in range(3)]
    if not all(np.isfinite(v) for v in p) or min(p) < T(0) or max(p) > T(1):
        return T(np.nan), [T(np.nan)] * 3, 0
    r = [T(0)] * 4

    def level(values, pp, d, out, direct):
        n = 1 << d
        nn = T(n)
        t = [pp[a] * nn for a in range(3)]
        cell = [min(max(int(np.ceil(t[a])) - 1, 0), n - 1) for a in range(3)]
        base = cell if direct else [int(np.floor(t[a])) for a in range(3)]
        fr = [t[a] - T(base[a]) for a in range(3)]
        for corner in range(8):
            cc = [corner // 4, (corner // 2) % 2, corner % 2]
            node = [cell[a] + cc[a] for a in range(3)]
            if not direct and min(node[a] - base[a] for a in range(3)) < 0:
                continue
            j = find(d, *node)
            if j < 0:
                continue
            hh, sg = [T(1) - fr[a] for a in range(3)], [T(-1)] * 3
            for a in range(3):
                if (cc[a] != 0) if direct else (node[a] > base[a]):
                    hh[a], sg[a] = fr[a], T(1)
            c = values[j]
            out[0] = out[0] + c * hh[0] * hh[1] * hh[2]
            if direct:
                cn = c * nn
                out[1] = out[1] + cn * (sg[0] * hh[1] * hh[2])
                out[2] = out[2] + cn * (hh[0] * sg[1] * hh[2])
                out[3] = out[3] + cn * (hh[0] * hh[1] * sg[2])
            else:
                out[1] = out[1] + c * nn * sg[0] * hh[1] * hh[2]
                out[2] = out[2] + c * nn * hh[0] * sg[1] * hh[2]
                out[3] = out[3] + c * nn * hh[0] * hh[1] * sg[2]

    if cum is None:
        for d in range(depth + 1):
            level(coeff, p, d, r, True)
    else:
        leaf = 0
        for d in range(depth, -1, -1):
            n = 1 << d
            c = [min(max(int(np.ceil(p[a] * T(n))) - 1, 0), n - 1) for a in range(3)]
            if find(d, *c) >= 0:
                leaf = d
                break
        p = [T(1e-6) if v == T(0) else (T(1.0 - 1e-6) if v == T(1) else v) for v in p]
        level(coeff, p, leaf, r, False)
        if leaf > 0:
            s = [T(0)] * 4
            level(cum, p, leaf - 1, s, False)
            r = [r[a] + s[a] for a in range(4)]
        if leaf < depth:
            s = [T(0)] * 4
            level(coeff, p, leaf + 1, s, False)
            r = [r[a] + s[a] for a in range(4)]
    grad = [(L[a] * r[1] + L[3 + a] * r[2]) + L[6 + a] * r[3] for a in range(3)]
    return r[0], grad, 1


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("reference", [False, True])
def test_adaptive_field_matches_restatement(user_lib, dtype, reference):
    T = np.dtype(dtype).type
    keys = adaptive_keys()
    coeff = np.random.default_rng(271).normal(size=len(keys)).astype(dtype)
    cum = cumulative_of(keys, coeff, T) if reference else None
    linear = (0., .5, 0., 0., 0., .5, .5, 0., 0.)
    translation = (.25, .25, .25)
    cube = np.concatenate([np.random.default_rng(2026).uniform(0, 1, (57, 3)),
                           [[0, .3, .4], [1, .3, .4], [.5, .3, .4], [.25, .3, .4], [.75, .3, .4],
                            [.5 - 1e-5, .3, .4], [.5 + 1e-5, .3, .4], [0, 0, 0], [1, 1, 1],
                            [1.01, .3, .4], [np.nan, .3, .4], [np.inf, .3, .4], [-np.inf, .3, .4]]])
    model = ((cube - .25) * 2)[:, [2, 0, 1]].astype(dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    d_keys = torch.tensor(keys, device="cuda")
    d_coeff = torch.tensor(coeff, device="cuda")
    d_cum = torch.tensor(cum, device="cuda") if reference else None
    handle = _lib.FieldHandle()
    handle.keys = d_keys.data_ptr()
    handle.coefficients = d_coeff.data_ptr()
    handle.cumulative = d_cum.data_ptr() if reference else None
    handle.count = len(keys)
    handle.linear[:] = linear
    handle.translation[:] = translation
    handle.depth = 2
    handle.dtype = _lib.PSR_FLOAT64 if dtype == np.float64 else _lib.PSR_FLOAT32
    values, gradients, valid = (t.cpu().numpy() for t in user_query(user_lib, handle,
                                                                     torch.tensor(model, dtype=tdt, device="cuda")))
    for i, q in enumerate(model):
        v, g, ok = restated_query(keys, coeff, cum, 2, linear, translation, q, T)
        assert valid[i] == ok, i
        np.testing.assert_array_equal(values[i], v, err_msg=str(i))
        np.testing.assert_array_equal(gradients[i], np.array(g, dtype), err_msg=str(i))
    np.testing.assert_array_equal(valid[-4:], 0)
    assert np.isnan(values[-4:]).all()
