// cli_convert.cpp -- bin/excent_convert (graph_tools.cpp).
#include "excent_b200.h"

int main(int argc, char** argv) { return excent_convert_main(argc, argv); }
