// reader_check.cpp - TEST-ONLY driver of the product's FASTA / FASTQ reader
// (poa_b200/csrc/reader.cpp): prints each record of a file as
// "name<TAB>comment<TAB>seq" so the tests can compare it with kseq's
// semantics (tests/fasta.py) on plain, gzip, FASTQ and CRLF inputs.
#include <cstdio>
#include <string>

#include "reader.h"

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    std::string text;
    if (!pb::read_file(argv[1], text)) return 1;
    for (const pb::SeqRec& r : pb::parse_fastx(text))
        std::printf("%s\t%s\t%s\n", r.name.c_str(), r.comment.c_str(), r.seq.c_str());
    return 0;
}
