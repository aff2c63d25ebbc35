// mld_mmio.h -- MatrixMarket I/O of a level hierarchy in the file layout of
// the reference's prec%dump (see mld_mmio.cpp for the file names).
#pragma once
#include <string>
#include <vector>

#include "mld_hier.h"

namespace mld {

bool file_exists(const std::string &f);
// <prefix><part>_p000_l<level, 3 digits>_<what>.mtx
std::string dump_name(const std::string &prefix, const char *part, int level, const char *what);

int read_mm_csr(const std::string &fname, CSR &a, std::string &msg);
int write_mm_csr(const std::string &fname, const CSR &a, const std::string &head, std::string &msg);
int read_mm_vec(const std::string &fname, std::vector<double> &v, std::string &msg);
int write_mm_vec(const std::string &fname, const std::vector<double> &v, const std::string &head,
                 std::string &msg);

// every level's coarse matrix, maps and smoother data
int dump_hierarchy(const std::vector<Level> &lv, const std::string &prefix, std::string &msg);
// nlev levels: level 1 matrix a0 (not part of a dump), the rest and the
// smoother data from files; the smoother kind of each level follows from the
// files present; sweeps and damping from p
int load_hierarchy(const std::string &prefix, int nlev, const CSR &a0, const Parms &p, std::vector<Level> &lv,
                   std::string &msg);

}  // namespace mld
