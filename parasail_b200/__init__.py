"""parasail-b200: Python access to the drop-in parasail.h library.

Attributes of this package (lib, align, batch_db, ...) come from
`parasail_b200.api`, which loads `libparasail_b200.so` the first time one of
them is read. Importing the package, or its submodule `synth` (the seeded
workload generators), maps no native code, so a process that only generates
inputs -- e.g. one that times a CPU implementation -- never loads the GPU
library.
"""
import importlib

_SUBMODULES = ("api", "synth", "tune")


def __getattr__(name):
    if name.startswith("__") or name in _SUBMODULES:
        raise AttributeError(name)
    api = importlib.import_module(".api", __name__)
    try:
        return getattr(api, name)
    except AttributeError:
        raise AttributeError("module 'parasail_b200' has no attribute %r" % name) from None
