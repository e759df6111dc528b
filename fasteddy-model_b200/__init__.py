"""B200-native FastEddy hot path: HYDRO_CORE tendency pipeline + RK3 stage commit.

Native code does the work (libfe_engine.so: sm_100a CUDA kernels; libfe_host.so: the
host C layer; libfe_refabi.so: the reference-named drop-in entry points). This package
only builds and binds them. The directory name has a hyphen, so import it with
importlib.import_module("fasteddy-model_b200").
"""
from . import build, cases, halo, runtime  # noqa: F401
from .runtime import Domain, Ensemble, FeConfig, FeError, Host, Mlp, load, read_binary  # noqa: F401

__all__ = ["build", "cases", "halo", "runtime", "Domain", "Ensemble", "FeConfig", "FeError", "Host", "Mlp", "load", "read_binary"]
