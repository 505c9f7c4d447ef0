// Instantiations of the thread-per-run kernel: VERIFY=false, SLOTS=true, every
// combination of 8-bit locations, global run state and race classes.
#include "sim_serial.cuh"

namespace csmc {
#define CSMC_SERIAL_INST(L8, GS, CL)                                                                      \
    template int serial_launch_one<false, true, L8, GS, CL>(const SimParams &, int, int, size_t, void *); \
    template int serial_occupancy_one<false, true, L8, GS, CL>(int, size_t, int *);
CSMC_SERIAL_INST(false, false, false)
CSMC_SERIAL_INST(false, true, false)
CSMC_SERIAL_INST(true, false, false)
CSMC_SERIAL_INST(true, true, false)
CSMC_SERIAL_INST(false, false, true)
CSMC_SERIAL_INST(false, true, true)
CSMC_SERIAL_INST(true, false, true)
CSMC_SERIAL_INST(true, true, true)
#undef CSMC_SERIAL_INST
}  // namespace csmc
