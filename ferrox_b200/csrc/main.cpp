// main.cpp -- the ferrox_b200 executable: `ferrox_b200 <inputs>`.
//
// Stands in for the reference's `main3d.gnu.*.ex inputs` (Source/main.cpp:35-46):
// same inputs keys, the same progress lines ("Advanced step N in T seconds",
// the steady-state norm, the sweep messages) and pltNNNNNNNN plotfiles at
// plot_int.  Extra keys may follow the file on the command line as
// key=value pairs, as AMReX ParmParse allows.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "../../include/ferrox_b200.h"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <inputs> [key=value ...]\n", argv[0]);
        return 2;
    }
    std::ifstream f(argv[1]);
    if (!f) {
        std::fprintf(stderr, "cannot open %s\n", argv[1]);
        return 2;
    }
    std::stringstream ss;
    ss << f.rdbuf() << "\n";
    for (int a = 2; a < argc; ++a) ss << argv[a] << "\n";
    ss << "fx.verbose = 1\n";
    fx_ctx* ctx = nullptr;
    int rc = fx_create(ss.str().c_str(), 1, &ctx);
    if (rc) {
        std::fprintf(stderr, "ferrox_b200: %s\n", fx_create_error());
        return 1;
    }
    int n[3];
    double dx[3];
    fx_get_dims(ctx, n, dx);
    std::printf("\n##### GEOMETRY PROPERTIES #####\n\n##### n_cell: %d  %d  %d\n", n[0], n[1], n[2]);
    double sc = 0;
    fx_get_param(ctx, "contains_sc", &sc);
    std::printf("contains_SC = %d\n", (int)sc);
    std::printf("\n ========= Advance Steps  ========== \n\n");
    int done = 0;
    rc = fx_run(ctx, &done);
    if (rc) {
        std::fprintf(stderr, "ferrox_b200: step %d: %s\n", done + 1, fx_last_error(ctx));
        fx_destroy(ctx);
        return 1;
    }
    fx_stats st;
    fx_get_stats(ctx, &st);
    std::printf("Steps: %d, V-cycles: %lld, Newton passes: %lld, device memory %.1f MB\n", st.step,
                st.mg_cycles_total, st.newton_iters_total, st.device_bytes / 1048576.0);
    fx_destroy(ctx);
    return 0;
}
