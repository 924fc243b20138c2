// Thin executables BP5, BP6, BK5, BK6: main() forwards to the library driver,
// which keeps the reference's command-line keys and result line.
#include "../include/bp_b200.h"

#ifndef BP_APP_NAME
#error "BP_APP_NAME must name the driver (BP5, BP6, BK5 or BK6)"
#endif

int main(int argc, char** argv) { return bp_driver_main(BP_APP_NAME, argc, argv) == BP_SUCCESS ? 0 : 1; }
