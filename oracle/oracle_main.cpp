// CPU ORACLE -- test infrastructure only (see oracle.h).  main.rs restated.
#include "oracle.h"
int main(int argc, char** argv) { return oracle::cli_main(argc, argv); }
