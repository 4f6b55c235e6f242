// sketch_harness.cpp - prints the minimizers that the UNMODIFIED reference's
// mm_sketch (src/minimizer.cpp:60-135, compiled into oracle/_ref/libminipoa.a)
// finds in each input line. TEST INFRASTRUCTURE: it pins the minimizer
// restatement that checks the band proposer's device feature kernel.
//
// Usage: sketch_harness K W < sequences (one per line)
// Output: one line per minimizer: <line index> <last base position> <hash>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "minimizer.h"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: sketch_harness K W < seqs\n");
        return 2;
    }
    const int k = std::atoi(argv[1]), w = std::atoi(argv[2]);
    std::string line;
    uint32_t rid = 0;
    while (std::getline(std::cin, line)) {
        mm128_v v = {0, 0, 0};
        mm_sketch(nullptr, line.c_str(), (int)line.size(), w, k, rid, 0, &v);
        for (size_t i = 0; i < v.n; i++)
            std::printf("%u %u %llu\n", rid, (unsigned)((uint32_t)v.a[i].y >> 1),
                        (unsigned long long)(v.a[i].x >> 8));
        std::free(v.a);
        rid++;
    }
    return 0;
}
