// plotfile.cpp -- single-level AMReX plotfile writer.
//
// Writes what WriteSingleLevelPlotfile produces for FerroX's plot MultiFab
// (Source/Plotfile.cpp:30, :177): a directory pltNNNNNNNN holding
//   Header              -- "HyperCLaw-V1.1", variable names, geometry, one box
//   Level_0/Cell_H      -- VisMF header: box array, FAB offsets, min/max
//   Level_0/Cell_D_00000-- "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))<box> <ncomp>\n"
//                          followed by ncomp x npts little-endian doubles, x fastest
// The format follows AMReX's published plotfile description; AMReX itself is
// not used.
#include "plotfile.h"

#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <sstream>

namespace fx {

namespace {

bool mkdir_p(const std::string& d) {
    if (d.empty()) return true;
    struct stat st;
    if (stat(d.c_str(), &st) == 0) return S_ISDIR(st.st_mode);
    size_t pos = d.find_last_of('/');
    if (pos != std::string::npos && pos > 0 && !mkdir_p(d.substr(0, pos))) return false;
    return mkdir(d.c_str(), 0755) == 0 || errno == EEXIST;
}

std::string box_str(const int n[3]) {
    std::ostringstream o;
    o << "((0,0,0) (" << n[0] - 1 << "," << n[1] - 1 << "," << n[2] - 1 << ") (0,0,0))";
    return o.str();
}

}  // namespace

std::string plotfile_name(int step) {
    std::ostringstream o;
    o << "plt" << std::setw(8) << std::setfill('0') << step;
    return o.str();
}

int write_plotfile(const std::string& dir, const PlotGeom& g, const std::vector<std::string>& names,
                   const std::vector<const double*>& comps, std::string* err) {
    const std::string lev = dir + "/Level_0";
    if (!mkdir_p(lev)) { if (err) *err = "cannot create " + lev; return -1; }
    const size_t npts = (size_t)g.n[0] * g.n[1] * g.n[2];
    const int ncomp = (int)comps.size();

    // data file
    std::vector<double> mn(ncomp), mx(ncomp);
    {
        std::ofstream f(lev + "/Cell_D_00000", std::ios::binary);
        if (!f) { if (err) *err = "cannot write " + lev + "/Cell_D_00000"; return -1; }
        f << "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))" << box_str(g.n) << " " << ncomp << "\n";
        for (int c = 0; c < ncomp; ++c) {
            const double* a = comps[c];
            double lo = a[0], hi = a[0];
            for (size_t q = 0; q < npts; ++q) { lo = std::min(lo, a[q]); hi = std::max(hi, a[q]); }
            mn[c] = lo; mx[c] = hi;
            f.write(reinterpret_cast<const char*>(a), (std::streamsize)(npts * sizeof(double)));
        }
        if (!f) { if (err) *err = "short write in Cell_D_00000"; return -1; }
    }
    // VisMF header
    {
        std::ofstream f(lev + "/Cell_H");
        if (!f) { if (err) *err = "cannot write Cell_H"; return -1; }
        f << "1\n0\n" << ncomp << "\n0\n";
        f << "(1 0\n" << box_str(g.n) << "\n)\n";
        f << "1\nFabOnDisk: Cell_D_00000 0\n\n";
        f.setf(std::ios::scientific, std::ios::floatfield);
        f.precision(15);
        f << "1," << ncomp << "\n";
        for (int c = 0; c < ncomp; ++c) f << mn[c] << ",";
        f << "\n\n1," << ncomp << "\n";
        for (int c = 0; c < ncomp; ++c) f << mx[c] << ",";
        f << "\n";
    }
    // plotfile header
    {
        std::ofstream f(dir + "/Header");
        if (!f) { if (err) *err = "cannot write Header"; return -1; }
        f.precision(17);
        f << "HyperCLaw-V1.1\n" << ncomp << "\n";
        for (auto& s : names) f << s << "\n";
        f << 3 << "\n" << g.time << "\n" << 0 << "\n";
        for (int d = 0; d < 3; ++d) f << g.prob_lo[d] << ' ';
        f << "\n";
        for (int d = 0; d < 3; ++d) f << g.prob_hi[d] << ' ';
        f << "\n\n";
        f << box_str(g.n) << " \n";
        f << g.step << " \n";
        for (int d = 0; d < 3; ++d) f << g.dx[d] << ' ';
        f << "\n0\n0\n";
        f << 0 << ' ' << 1 << ' ' << g.time << "\n" << g.step << "\n";
        for (int d = 0; d < 3; ++d) f << g.prob_lo[d] << ' ' << g.prob_lo[d] + g.n[d] * g.dx[d] << "\n";
        f << "Level_0/Cell\n";
    }
    return 0;
}

}  // namespace fx
