// main_cli.cpp -- the pfc-exp-cli executable: a thin wrapper over pfc_run_cli()
// (the reference's entry point is src/experiment/main_cli.cpp:24-88).
#include "pfc_b200.h"

int main(int argc, char **argv) { return pfc_run_cli(argc, argv); }
