"""relaxmap_b200: RelaxMap's map-equation optimiser on one B200 (sm_100a).

The engine is librelaxmap_b200.so (C ABI, include/relaxmap_b200.h) with the
drop-in command line relaxmap_b200/ompRelaxmap; this package is its Python
binding (ctypes) plus seeded synthetic graph generators.
"""
from ._lib import (EXPORTS, LIB_PATH, TUNING_FIELDS, Batch, Graph, Opts, RmxError, cli, default_opts, get_tuning,
                   lib, parse_file, read_clu, release_device_cache, set_tuning)

__all__ = ["Batch", "Graph", "Opts", "RmxError", "cli", "default_opts", "lib", "LIB_PATH", "EXPORTS", "parse_file",
           "release_device_cache", "get_tuning", "set_tuning", "TUNING_FIELDS", "read_clu"]
