// omicabelnomm CLI: the reference's command line (src/main.cpp) on the B200 engine.
#include "omicabel_b200.h"

int main(int argc, char** argv) { return oa_cli_main(argc, argv); }
