"""The subset objective as a torch autograd function (libtorch C++ extension
dice_b200/torch_ext/dicegpu_autograd.cpp over libdicegpu.so's
dicegpu_adjoint).

    from dice_b200 import autograd
    gamma = autograd.subset_objective(params, def_image, schema)   # n values
    gamma.sum().backward()   # d/dparams (n x 6 or 12) and d/ddef_image (H x W)

`build()` compiles the extension in-tree (dice_b200/torch_ext/_build); at
run time the built module is imported from there, and its absence is an
error (there is no Python fallback).
"""
import importlib.machinery
import importlib.util
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "torch_ext", "dicegpu_autograd.cpp")
_BUILD = os.path.join(_HERE, "torch_ext", "_build")
_NAME = "dicegpu_autograd"
_mod = None


def build(verbose=False):
    """Compiles the extension into dice_b200/torch_ext/_build (needs
    libdicegpu.so built first: it links against it)."""
    from torch.utils import cpp_extension
    from dice_b200 import abi
    abi.load_library()   # the import at the end of the build resolves it by soname
    os.makedirs(_BUILD, exist_ok=True)
    inc = os.path.join(os.path.dirname(_HERE), "include")
    # the run path is the package directory, two levels above the built
    # module: "$$" is ninja's escape for "$", the quotes keep the shell that
    # runs the link from expanding $ORIGIN
    cpp_extension.load(name=_NAME, sources=[_SRC], extra_include_paths=[inc],
                       extra_cflags=["-O2"],
                       extra_ldflags=["-L" + _HERE, "-ldicegpu", "-Wl,-rpath,'$$ORIGIN/../..'"],
                       with_cuda=True, build_directory=_BUILD, verbose=verbose)
    return os.path.join(_BUILD, _NAME + ".so")


def load():
    """Imports the built extension (libdicegpu.so is loaded first by the ABI
    module, so both share one copy of the library)."""
    global _mod
    if _mod is None:
        import torch  # noqa: F401  (the extension needs libtorch loaded)
        from dice_b200 import abi
        abi.load_library()
        path = os.path.join(_BUILD, _NAME + ".so")
        if not os.path.exists(path):
            raise RuntimeError("%s is not built; run __graft_entry__.build()" % path)
        loader = importlib.machinery.ExtensionFileLoader(_NAME, path)
        spec = importlib.util.spec_from_file_location(_NAME, path, loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        _mod = mod
    return _mod


def subset_objective(params, def_image, schema, objective=0):
    """Per-subset objective of `schema`'s subsets (0: gamma, 1: Gauss-Newton
    least squares) at `params` (n x 6 affine / n x 12 quadratic, CUDA) on
    `def_image` (H x W float32 CUDA), differentiable in both."""
    from dice_b200 import abi
    quadratic = schema.params.shape_function == abi.QUADRATIC_SF
    return load().subset_objective(params, def_image, int(schema.ctx.value), objective, quadratic)
