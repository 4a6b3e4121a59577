"""Recipe: build the reference's own per-node LLG/anisotropy kernels for the CPU.

TEST INFRASTRUCTURE.  The reference keeps its per-node kernels as CUDA-C
bodies inside ``cupy.ElementwiseKernel(...)`` calls
(``gpu/solvers/llg_module_GPU.py:100-308``,
``gpu/fields/Anisotropy_GPU.py:24-50``, ``gpu/solvers/llg_stt_module_GPU.py:101-393``,
``gpu/solvers/llg_SOT_module_GPU.py:170-437``).  Those bodies are plain C
arithmetic on doubles, so this recipe reads the reference sources where they
lie, pulls each kernel's parameter lists and body out of the Python AST, wraps
each body in a C loop over arrays and compiles the result with gcc into
``oracle/_ref/libref_elementwise.so``.  Nothing from the reference is copied
into the repository: the generated C file and the library live only under
``oracle/_ref/`` (git-ignored).  The library is used to make the golden fixtures
under ``tests/golden/`` (``make_golden.py``); the tests read those fixtures, so they
run where the reference checkout is absent.

The reference's CPU Jv kernel (``cpu/solvers/llg_module.py:25-74``) is a numba
function inside a module that needs DOLFINx to import; ``load_cpu_jv`` pulls
just that function out of the AST and JIT-compiles it with numba.
"""
from __future__ import annotations

import ast
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

# The reference checkout this recipe reads: $SPX_REFERENCE_PATH, by default the
# read-only checkout beside the build container's repository.
REF_ROOT = Path(os.environ.get("SPX_REFERENCE_PATH", "/root/reference")) / "src" / "spinfemx"
HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"

KERNELS = {
    "_LLG_RHS_KERNEL": "gpu/solvers/llg_module_GPU.py",
    "_JAC_VEC_KERNEL": "gpu/solvers/llg_module_GPU.py",
    "_PC_BUILD_INV3_KERNEL": "gpu/solvers/llg_module_GPU.py",
    "_PC_APPLY_KERNEL": "gpu/solvers/llg_module_GPU.py",
    "_ANISOTROPY_NODAL_KERNEL": "gpu/fields/Anisotropy_GPU.py",
    "_ANISOTROPY_DIAG_KERNEL": "gpu/fields/Anisotropy_GPU.py",
    "_LLG_RHS_STT_KERNEL": "gpu/solvers/llg_stt_module_GPU.py",
    "_JAC_VEC_STT_KERNEL": "gpu/solvers/llg_stt_module_GPU.py",
    "_PC_BUILD_INV3_STT_KERNEL": "gpu/solvers/llg_stt_module_GPU.py",
    "_LLG_RHS_SOT_KERNEL": "gpu/solvers/llg_SOT_module_GPU.py",
    "_JAC_VEC_SOT_KERNEL": "gpu/solvers/llg_SOT_module_GPU.py",
    "_PC_BUILD_INV3_SOT_KERNEL": "gpu/solvers/llg_SOT_module_GPU.py",
}

_CTYPE = {"float64": "double", "int32": "int"}


def _extract(path: Path, name: str):
    tree = ast.parse(path.read_text())
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(
                isinstance(t, ast.Name) and t.id == name for t in node.targets):
            call = node.value
            args = [ast.literal_eval(a) for a in call.args[:3]]
            return args[0], args[1], args[2]
    raise KeyError(name)


def _params(spec: str):
    out = []
    for item in spec.split(","):
        item = item.strip()
        if not item:
            continue
        t, n = item.split()
        out.append((_CTYPE[t], n))
    return out


def kernel_signatures():
    sigs = {}
    for name, rel in KERNELS.items():
        ins, outs, body = _extract(REF_ROOT / rel, name)
        sigs[name] = (_params(ins), _params(outs), body)
    return sigs


def build(force: bool = False) -> Path:
    """Compile the extracted kernel bodies; returns the library path."""
    REF_OUT.mkdir(parents=True, exist_ok=True)
    lib = REF_OUT / "libref_elementwise.so"
    if lib.exists() and not force:
        return lib
    sigs = kernel_signatures()
    src = ["#include <math.h>", ""]
    for name, (ins, outs, body) in sigs.items():
        # every parameter is passed as an array; scalars are broadcast via stride 0
        plist = [f"const {t}* __in_{n}, long __s_{n}" for t, n in ins]
        plist += [f"{t}* __out_{n}" for t, n in outs]
        src.append(f"void ref{name}(long __n, {', '.join(plist)}) {{")
        src.append("  for (long __i = 0; __i < __n; ++__i) {")
        for t, n in ins:
            src.append(f"    const {t} {n} = __in_{n}[__i * __s_{n}];")
        for t, n in outs:
            src.append(f"    {t} {n};")
        src.append("    {")
        src.append(body)
        src.append("    }")
        for t, n in outs:
            src.append(f"    __out_{n}[__i] = {n};")
        src.append("  }")
        src.append("}")
        src.append("")
    c_file = REF_OUT / "ref_elementwise.c"
    c_file.write_text("\n".join(src))
    subprocess.check_call(["gcc", "-O2", "-fno-fast-math", "-ffp-contract=off", "-shared",
                           "-fPIC", "-o", str(lib), str(c_file), "-lm"])
    return lib


class RefElementwise:
    """ctypes front-end: ``call(name, n, inputs: dict, ) -> dict of outputs``."""

    def __init__(self, lib_path=None):
        self.lib = ctypes.CDLL(str(lib_path or build()))
        self.sigs = kernel_signatures()

    def call(self, name, n, inputs):
        ins, outs, _ = self.sigs[name]
        fn = getattr(self.lib, "ref" + name)
        args = [ctypes.c_long(n)]
        keep = []
        for t, pname in ins:
            val = inputs[pname]
            dt = np.float64 if t == "double" else np.int32
            arr = np.ascontiguousarray(np.atleast_1d(np.asarray(val, dtype=dt)))
            keep.append(arr)
            args += [arr.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(0 if arr.size == 1 else 1)]
        res = {}
        for t, pname in outs:
            arr = np.empty(n, dtype=np.float64 if t == "double" else np.int32)
            res[pname] = arr
            args.append(arr.ctypes.data_as(ctypes.c_void_p))
        fn(*args)
        return res


def load_cpu_jv():
    """numba-compiled jac_vec_local_kernel from cpu/solvers/llg_module.py:25-74."""
    import math  # noqa: F401  (available to the exec'd source)
    from numba import njit
    path = REF_ROOT / "cpu/solvers/llg_module.py"
    text = path.read_text()
    tree = ast.parse(text)
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name == "jac_vec_local_kernel":
            node.decorator_list = []
            mod = ast.Module(body=[node], type_ignores=[])
            ns = {}
            exec(compile(mod, str(path), "exec"), ns)
            return njit(fastmath=True)(ns["jac_vec_local_kernel"])
    raise KeyError("jac_vec_local_kernel")


def import_reference_hmatrix():
    """Import lindholm_hmatrix_gpu submodules and Lindholm_kernel without DOLFINx."""
    import importlib
    import sys
    import types
    pkg_dir = REF_ROOT / "gpu/fields/lindholm_hmatrix_gpu"
    name = "_spx_ref_hmat"
    if name not in sys.modules:
        pkg = types.ModuleType(name)
        pkg.__path__ = [str(pkg_dir)]
        sys.modules[name] = pkg
    mods = {}
    for sub in ("tree", "lindholm_kernel", "entry_provider", "compressors", "storage", "builder"):
        mods[sub] = importlib.import_module(f"{name}.{sub}")
    spec = importlib.util.spec_from_file_location(
        "_spx_ref_lindholm_kernel", REF_ROOT / "gpu/fields/Lindholm_kernel.py")
    lk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(lk)
    mods["Lindholm_kernel"] = lk
    return mods


if __name__ == "__main__":
    print(build(force=True))
    os.environ.setdefault("NUMBA_NUM_THREADS", str(os.cpu_count()))
