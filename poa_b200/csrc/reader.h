// reader.h - FASTA / FASTQ input as minipoa reads it (src/handle_input.cpp:
// 13-43: kseq over gzread, so plain or gzip-compressed files): per record the
// name up to the first blank, the rest of the header line as the comment,
// and the sequence lines joined; FASTQ quality lines are skipped.
#pragma once
#include <string>
#include <vector>

namespace pb {

struct SeqRec {
    std::string name, comment, seq;
};

// The whole file, decompressed when it is gzip; false when it cannot be read.
bool read_file(const char* path, std::string& out);
std::vector<SeqRec> parse_fastx(const std::string& text);

}  // namespace pb
