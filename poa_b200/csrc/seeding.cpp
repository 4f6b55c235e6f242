// seeding.cpp - placeholder until the minimizer seeding restatement lands:
// the driver refuses -S and -p before reaching these.
#include "seeding.h"

#include "driver.h"

namespace pb {

void Seeder::init(const Params&, const std::vector<std::string>& seqs) {
    nseq_ = (int)seqs.size();
    ord.resize(nseq_);
    rid_to_ord.resize(nseq_);
    for (int i = 0; i < nseq_; i++) ord[i] = rid_to_ord[i] = i;
}
void Seeder::guide_tree(const Params&) {}
void Seeder::anchors_by_consensus(const Params&, int, int, const std::string&, std::vector<Anchor>& out) { out.clear(); }

}  // namespace pb
