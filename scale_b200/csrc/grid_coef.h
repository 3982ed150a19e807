// Host-side coefficient tables (see grid_coef.cpp).
#pragma once
#include <vector>

namespace hevi {

void build_f2h(int KA, const double *CDZ, double *F2H1, double *F2H2);

struct NdGrid {
    int KA, IA, JA, KS, KE, IS, IE, JS, JE;
    const double *CDZ, *FDZ, *CDX, *FDX, *CDY, *FDY;
};
struct NdTables {
    std::vector<double> CNZ3, CNX3, CNY3, cdz, fdz, cdx, fdx, cdy, fdy;
    std::vector<double> CNZ4, CNX4, CNY4; // (5,KA,2) (5,IA,2) (5,JA,2), for ND_ORDER > 1
};
void build_nd_tables(const NdGrid &gr, double DT, double ND_COEF, int ND_ORDER, NdTables &t);

}  // namespace hevi
