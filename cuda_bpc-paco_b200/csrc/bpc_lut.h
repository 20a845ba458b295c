// bpc_lut.h -- host LUT loader (load_LUTs semantics, main_example.cu:219-448).
#pragma once
#include <vector>

namespace bpc {

constexpr int kErrArg = -1;
constexpr int kErrCuda = -2;
constexpr int kErrFile = -3;
constexpr int kErrParse = -4;
constexpr int kErrNoMem = -5;

long lut_section_size(int max_bitplane, int nctx, int levels);
long lut_entries(int passes, int levels, int max_bitplane);
// Loads a LUT folder (a path prefix ending in '/') into `lut`.  0 or kErr*.
int load_luts_host(const char *folder, int passes, int levels, std::vector<int> &lut);

}  // namespace bpc
