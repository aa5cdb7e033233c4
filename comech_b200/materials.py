"""Material mixing of the engine's cells on the device, with the reference's entry point and results:
``materials(V, roles, cart_E, nu_soft) -> (E, nu, active, F, ser)`` of rb/rbfe.py:75-134.

The class list and the material table are the engine's (rb/rbgeom.py:45-50): the mixing rule is defined on
them, so they are the same here.  The work runs in libfeb200.so (``feb_mix_materials``); no CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _lib
from .engine import _dev, _host, _ptr, _stream, _torch

CLASSES = ["void", "cortical", "cancellous", "cartilage", "fascia", "soft", "plate", "fibrous", "fat", "gap"]
MAT = {"cortical": (7300.0, 0.3), "cancellous": (100.0, 0.3), "cartilage": (10.0, 0.4), "fascia": (350.0, 0.4),
       "soft": (1.15, 0.49), "plate": (17000.0, 0.1), "fibrous": (60.0, 0.4), "fat": (1.15, 0.45), "gap": (0.01, 0.3)}


def bone_groups(cls, roles):
    """Group id (1..) per bone body: the named bones of ``roles`` in order, then every other cortical /
    cancellous body on its own, except ``roles['bonded_extra']`` (rb/replica2.py:34-46)."""
    g, names, k = {}, {}, 1
    for name, bodies in roles["bones"].items():
        for b in bodies:
            g[b] = k
        names[k] = name
        k += 1
    skip = set(roles.get("bonded_extra", ()))
    for b, c in sorted(cls.items()):
        if c in (1, 2) and b not in g and b not in skip:
            g[b] = k
            names[k] = f"body{b}"
            k += 1
    return g, names


def class_table(cart_E=10.0, nu_soft=0.49):
    """Per-class lambda, mu and lambda + 2 mu of the mixing rule (rb/rbfe.py:85-88)."""
    mat = dict(MAT)
    mat["cartilage"] = (cart_E, 0.4)
    mat["soft"] = (1.15, nu_soft)
    E = np.array([1.0] + [mat[c][0] for c in CLASSES[1:]])
    nu = np.array([0.3] + [mat[c][1] for c in CLASSES[1:]])
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return lam, mu, lam + 2 * mu


def materials(V, roles, cart_E=10.0, nu_soft=0.49):
    """(E, nu, active, F, ser) of every cell of V (``cls``: body -> class, ``L``: ncell x ns^3 body labels,
    ``xe ye ze``) under ``roles`` (``bones``: name -> bodies, ``bonded_extra``), as rb/rbfe.py:75-134."""
    torch = _torch()
    cls = {int(k): int(v) for k, v in V["cls"].items()}
    L = np.asarray(V["L"])
    nb = max(max(cls), int(L.max()))
    body_class = np.zeros(nb + 1, np.int8)
    for b, c in cls.items():
        if not 0 <= c < len(CLASSES):
            raise ValueError(f"body {b}: class {c} outside 0..{len(CLASSES) - 1}")
        body_class[b] = c
    grp, _ = bone_groups(cls, roles)
    if grp and max(grp.values()) > 64:
        raise ValueError("more than 64 bone groups")
    body_group = np.zeros(nb + 1, np.int8)
    for b, k in grp.items():
        if 0 <= b <= nb:
            body_group[b] = k
    nx, ny, nz = len(V["xe"]) - 1, len(V["ye"]) - 1, len(V["ze"]) - 1
    ncell = nx * ny * nz
    if L.shape[0] != ncell:
        raise ValueError("L needs one row per cell")
    lam, mu, M = (np.ascontiguousarray(a, np.float64) for a in class_table(cart_E, nu_soft))
    Ld = _dev(L.astype(np.int32), np.int32)
    bc = torch.from_numpy(body_class).cuda()
    bg = torch.from_numpy(body_group).cuda()
    F = torch.empty(ncell * len(CLASSES), dtype=torch.float64, device="cuda")
    E = torch.empty(ncell, dtype=torch.float64, device="cuda")
    nu = torch.empty(ncell, dtype=torch.float64, device="cuda")
    act = torch.empty(ncell, dtype=torch.uint8, device="cuda")
    ser = torch.empty(ncell, dtype=torch.uint8, device="cuda")
    _lib.check(_lib.load().feb_mix_materials(nx, ny, nz, L.shape[1], _ptr(Ld), nb + 1, _ptr(bc), _ptr(bg),
                                             lam.ctypes.data_as(C.c_void_p), mu.ctypes.data_as(C.c_void_p),
                                             M.ctypes.data_as(C.c_void_p), _ptr(F), _ptr(E), _ptr(nu), _ptr(act),
                                             _ptr(ser), _stream()))
    E_h, nu_h, a_h, F_h, s_h = _host(E, nu, act, F.view(ncell, len(CLASSES)), ser)
    return E_h, nu_h, a_h.astype(bool), F_h, s_h.astype(bool)
