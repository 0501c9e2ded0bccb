// Drop-in executable: the reference's command line on the B200 engine.
#include "../../include/relaxmap_b200.h"

int main(int argc, char **argv) { return rmx_cli_main(argc, argv); }
