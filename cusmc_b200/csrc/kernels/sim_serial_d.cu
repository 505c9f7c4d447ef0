// Instantiations of the thread-per-run kernel: VERIFY=true, SLOTS=true, every
// combination of 8-bit locations and global run state.
#include "sim_serial.cuh"

namespace csmc {
#define CSMC_SERIAL_INST(L8, GS)                                                                      \
    template int serial_launch_one<true, true, L8, GS>(const SimParams &, int, int, size_t, void *); \
    template int serial_occupancy_one<true, true, L8, GS>(int, size_t, int *);
CSMC_SERIAL_INST(false, false)
CSMC_SERIAL_INST(false, true)
CSMC_SERIAL_INST(true, false)
CSMC_SERIAL_INST(true, true)
#undef CSMC_SERIAL_INST
}  // namespace csmc
