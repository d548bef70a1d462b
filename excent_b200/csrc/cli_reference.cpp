// cli_reference.cpp -- bin/excent_reference: the FP64 oracle as a GPU tool, and dump comparison.
#include "excent_b200.h"

int main(int argc, char** argv) { return excent_reference_main(argc, argv); }
