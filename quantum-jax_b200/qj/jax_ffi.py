"""JAX binding: the reference's step and get_potential as XLA custom calls.

The reference runs ``jax.lax.fori_loop(0, nt_sub, update, state)``
(quantum-stars.py:454) with ``update`` calling ``compute_step``
(:295-330), and ``get_potential`` (:189-193) inside it.  With this module a
script keeps its jitted loop and replaces those two functions::

    from qj import jax_ffi
    jax_ffi.register()
    psi, pos, vel, diag = jax_ffi.kdk_step(psi, pos, vel, diag, grid=grid, phys=phys,
                                           m_s=m_s, dt=dt, nsteps=nt_sub)
    V = jax_ffi.get_potential(rho, grid=grid, phys=phys)

Both lower to XLA custom calls (status-returning GPU form, api_version 2)
whose targets are exported by libqj.so (``qj_xla_kdk_step_f32``,
``qj_xla_get_potential_f32``; include/qj.h documents their buffers and
descriptors) and run on XLA's stream.  Arrays are complex64 / float32, as the
reference with x64 off.

jaxlib cannot be installed in the build environment of this repository, so
the JAX side (primitives, lowering, registration) is untested there; the
targets themselves are tested through ctypes with device-pointer arrays and
packed descriptors (``pack_kdk``, ``pack_poisson``), which is exactly what
XLA hands them.
"""

from __future__ import annotations

import ctypes

from . import _lib

KDK_TARGET = "qj_xla_kdk_step_f32"
POISSON_TARGET = "qj_xla_get_potential_f32"


def _grid(grid):
    return _lib.QjGrid(grid.nx, grid.ny, grid.nz, grid.Lx, grid.Ly, grid.Lz)


def _phys(p):
    return _lib.QjPhys(p.m_per_hbar, p.G, p.rho_bar, p.b_coeff, p.cs, p.c_light)


def pack_kdk(grid, phys, n_s, m_s, dt, nsteps, self_interaction=False, has_v_ext=False) -> bytes:
    """The backend_config (qj_xla_kdk_desc) of a kdk_step custom call."""
    d = _lib.QjXlaKdkDesc(_lib.QJ_XLA_DESC_VERSION, int(nsteps), int(n_s),
                          int(bool(self_interaction)), int(bool(has_v_ext)), 0, _grid(grid),
                          _phys(phys), float(m_s), float(dt))
    return bytes(d)


def pack_poisson(grid, phys, self_interaction=False) -> bytes:
    """The backend_config (qj_xla_poisson_desc) of a get_potential custom call."""
    d = _lib.QjXlaPoissonDesc(_lib.QJ_XLA_DESC_VERSION, int(bool(self_interaction)), _grid(grid),
                              _phys(phys))
    return bytes(d)


def _capsule(fn_ptr):
    """A PyCapsule named as XLA expects for a custom-call target."""
    new = ctypes.pythonapi.PyCapsule_New
    new.restype = ctypes.py_object
    new.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
    return new(fn_ptr, b"xla._CUSTOM_CALL_TARGET", None)


def _status_setter():
    """jaxlib's XlaCustomCallStatusSetFailure, if its extension exports it."""
    try:
        import jaxlib.xla_extension as xe

        f = ctypes.CDLL(xe.__file__).XlaCustomCallStatusSetFailure
        return ctypes.cast(f, ctypes.c_void_p).value
    except (ImportError, OSError, AttributeError):
        return None


_registered = False
_prims = {}


def register():
    """Register both targets with XLA for CUDA and define the primitives."""
    global _registered
    if _registered:
        return
    import jax
    from jax.interpreters import mlir

    try:
        from jax.extend.core import Primitive
    except ImportError:  # older JAX
        from jax.core import Primitive

    L = _lib.lib()
    fn = _status_setter()
    if fn:
        L.qj_xla_set_status_fn(ctypes.c_void_p(fn))
    for name in (KDK_TARGET, POISSON_TARGET):
        ptr = ctypes.cast(getattr(L, name), ctypes.c_void_p).value
        jax.ffi.register_ffi_target(name, _capsule(ptr), platform="CUDA", api_version=0)

    kdk = Primitive("qj_kdk_step")
    kdk.multiple_results = True
    kdk.def_abstract_eval(lambda psi, pos, vel, diag, *rest, **kw: (psi, pos, vel, diag))

    def kdk_lowering(ctx, psi, pos, vel, diag, *rest, opaque):
        outs = [mlir.aval_to_ir_type(a) for a in ctx.avals_out]
        return mlir.custom_call(KDK_TARGET, result_types=outs,
                                operands=[psi, pos, vel, diag, *rest], backend_config=opaque,
                                api_version=2,
                                operand_output_aliases={0: 0, 1: 1, 2: 2, 3: 3}).results

    mlir.register_lowering(kdk, kdk_lowering, platform="cuda")

    pot = Primitive("qj_get_potential")
    pot.def_abstract_eval(lambda rho, **kw: rho)

    def pot_lowering(ctx, rho, *, opaque):
        return mlir.custom_call(POISSON_TARGET,
                                result_types=[mlir.aval_to_ir_type(ctx.avals_out[0])],
                                operands=[rho], backend_config=opaque, api_version=2).results

    mlir.register_lowering(pot, pot_lowering, platform="cuda")
    _prims["kdk"], _prims["pot"] = kdk, pot
    _registered = True


def kdk_step(psi, pos, vel, diag, *, grid, phys, m_s, dt, nsteps, self_interaction=False,
             v_ext=None):
    """nsteps x compute_step (quantum-stars.py:295-330) inside a jitted program:
    psi complex64 [nx, ny, nz], pos / vel float32 [n_s, 3], diag float64 [3]
    (t, a_max, dt_s; needs jax_enable_x64 for the float64 diag, else pass it
    as float32 [3] and convert).  Returns the new (psi, pos, vel, diag)."""
    register()
    opaque = pack_kdk(grid, phys, pos.shape[0], m_s, dt, nsteps, self_interaction,
                      v_ext is not None)
    args = (psi, pos, vel, diag) + ((v_ext,) if v_ext is not None else ())
    return tuple(_prims["kdk"].bind(*args, opaque=opaque))


def get_potential(rho, *, grid, phys, self_interaction=False):
    """get_potential (quantum-stars.py:189-193): float32 rho -> V."""
    register()
    return _prims["pot"].bind(rho, opaque=pack_poisson(grid, phys, self_interaction))
