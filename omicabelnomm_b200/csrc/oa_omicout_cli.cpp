// omicout CLI: the reference's OmicOUT command line (OmicOUT/main.cpp) on this library.
#include "omicabel_b200.h"

int main(int argc, char** argv) { return oa_omicout_main(argc, argv); }
