// fastgrid4 / autogrid4 drop-in executable: the whole program is ag_main().
#include "../../include/fastgrid_b200.h"

int main(int argc, char** argv) { return ag_main(argc, argv); }
