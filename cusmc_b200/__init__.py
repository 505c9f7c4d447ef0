"""cusmc_b200: statistical model checking of stochastic timed automata on B200.

Drop-in for the simulation path of AndreasHolt/cuSMC: same UPPAAL models,
same queries, same reports; hand-written sm_100a kernels behind the C ABI in
include/csmc.h (libcsmc.so).
"""
from .api import (  # noqa: F401
    QUERY_LOCATION,
    QUERY_VARIABLE,
    Configuration,
    Network,
    Query,
    Result,
    StatisticsConfiguration,
    blob_info,
    compile_model,
    dump_model,
    location_query,
    make_query,
    run_host,
    smc,
    variable_query,
    version,
)
