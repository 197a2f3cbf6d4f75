/* Stand-in for parsb's SlashBurn.h so that the reference's src/class.cu
 * compiles without abseil/fmt/spray/ips4o (they need a network fetch).
 * Only the names class.cu mentions are declared; none of them is on the
 * reordered-SpMV path, and calling them aborts. Test infrastructure only. */
#ifndef MR_REF_STUB_SLASHBURN_H
#define MR_REF_STUB_SLASHBURN_H
#include <random>
#include <string>
#include <vector>
#include <cstdlib>
struct CLApp {
    CLApp(const std::string&, double, int) {}
    double percent() const { return 0.0; }
    int num_threads() const { return 1; }
};
struct Graph { long num_nodes() const { std::abort(); return 0; } };
struct Builder { explicit Builder(const CLApp&) {} Graph MakeGraph() { std::abort(); return Graph(); } };
struct Bitmap { explicit Bitmap(long) {} };
struct SlashBurn {
    std::vector<int> perm;
    SlashBurn(const Graph&, int, double, Bitmap&, int) { std::abort(); }
};
#endif
