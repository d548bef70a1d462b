// cli_evict.cpp -- bin/excent_evict (graph_tools.cpp).
#include "excent_b200.h"

int main(int argc, char** argv) { return excent_evict_main(argc, argv); }
