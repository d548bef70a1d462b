// cli_info.cpp -- bin/excent_info (graph_tools.cpp).
#include "excent_b200.h"

int main(int argc, char** argv) { return excent_info_main(argc, argv); }
