// gpe_main.cpp -- the `gpe` driver: `gpe <input file>` (main.cu:20-82).
#include <iostream>

#include "../../include/gpe_host.h"

int main(int argc, const char* argv[]) {
    if (argc != 2) {
        std::cerr << "Usage: " << argv[0] << " <filename>" << std::endl;
        return 1;
    }
    return gpeh_run(argv[1]);
}
