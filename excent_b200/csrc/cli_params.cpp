// cli_params.cpp -- bin/excent_params: the given constants of a graph (.env).
#include "excent_b200.h"

int main(int argc, char** argv) { return excent_params_main(argc, argv); }
