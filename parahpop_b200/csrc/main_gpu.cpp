// parahpop_gpu CONFIG.json TARGETS.json OUTPUT_DIRECTORY  (src/gpu/main.cpp:1-3)
#include "../../include/parahpop.h"

int main(int argc, char** argv) { return paraHPOP_run(argc, argv, "device"); }
