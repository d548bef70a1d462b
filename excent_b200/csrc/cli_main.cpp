// cli_main.cpp -- bin/excent: the command line, as the reference binary takes it.
#include "excent_b200.h"

int main(int argc, char** argv) { return excent_cli_main(argc, argv); }
