// reader.cpp - FASTA / FASTQ input as minipoa reads it (see reader.h).
#include "reader.h"

#include <zlib.h>

namespace pb {

bool read_file(const char* path, std::string& out) {
    gzFile fp = gzopen(path, "r");
    if (!fp) return false;
    char buf[1 << 16];
    int n;
    while ((n = gzread(fp, buf, sizeof(buf))) > 0) out.append(buf, (size_t)n);
    gzclose(fp);
    return n >= 0;
}

std::vector<SeqRec> parse_fastx(const std::string& s) {
    std::vector<SeqRec> recs;
    size_t i = 0, n = s.size();
    while (i < n) {
        if (s[i] != '>' && s[i] != '@') { i++; continue; }
        const bool fq = s[i] == '@';
        size_t eol = s.find('\n', i);
        if (eol == std::string::npos) eol = n;
        size_t he = eol;
        if (he > i + 1 && s[he - 1] == '\r') he--;
        const std::string hdr = s.substr(i + 1, he - i - 1);
        SeqRec r;
        const size_t sp = hdr.find_first_of(" \t");
        r.name = hdr.substr(0, sp);
        if (sp != std::string::npos) r.comment = hdr.substr(sp + 1);
        i = eol < n ? eol + 1 : n;
        while (i < n && s[i] != '>' && !(fq && s[i] == '+') && !(!fq && s[i] == '@')) {
            if (s[i] != '\n' && s[i] != '\r') r.seq.push_back(s[i]);
            i++;
        }
        if (fq && i < n && s[i] == '+') {
            const size_t e2 = s.find('\n', i);
            i = e2 == std::string::npos ? n : e2 + 1;
            size_t ql = 0;
            while (i < n && ql < r.seq.size()) {
                if (s[i] != '\n' && s[i] != '\r') ql++;
                i++;
            }
        }
        recs.push_back(std::move(r));
    }
    return recs;
}

}  // namespace pb
