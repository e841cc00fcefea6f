"""kushdb_b200: B200 execution backend for KushDB's relational hot path.

ScanSelect -> HashJoin -> GroupByAggregate -> OrderBy (+ SkinnerJoin) plans,
built with :mod:`kushdb_b200.plan`, run as generated sm_100a CUDA pipelines
over HBM-resident columns through the C ABI in ``include/kdb_b200.h``.
"""

from .data import HostColumn, HostTable, catalog_of, load_golden, read_kdb  # noqa: F401
from .plan import *  # noqa: F401,F403

__all__ = ["Engine", "HostColumn", "HostTable"]


def __getattr__(name):
    if name == "Engine":
        from .engine import Engine
        return Engine
    raise AttributeError(name)
