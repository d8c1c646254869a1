// plotfile.h -- single-level AMReX plotfile writer (Source/Plotfile.cpp output).
#pragma once

#include <string>
#include <vector>

namespace fx {

struct PlotGeom {
    int n[3];
    double prob_lo[3], prob_hi[3], dx[3];
    double time;
    int step;
};

std::string plotfile_name(int step);
int write_plotfile(const std::string& dir, const PlotGeom& g, const std::vector<std::string>& names,
                   const std::vector<const double*>& comps, std::string* err);

}  // namespace fx
