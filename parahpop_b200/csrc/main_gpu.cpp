// parahpop_gpu CONFIG.json TARGETS.json OUTPUT_DIRECTORY  (src/gpu/main.cpp:1-3)
// parahpop_gpu --serve SOCKET | --stop SOCKET: the resident environment server
#include <cstring>

#include "../../include/parahpop.h"

int main(int argc, char** argv) {
    if (argc == 3 && std::strcmp(argv[1], "--serve") == 0) return phop_resident_serve(argv[2], "device");
    if (argc == 3 && std::strcmp(argv[1], "--stop") == 0) return phop_resident_stop(argv[2]);
    return paraHPOP_run(argc, argv, "device");
}
