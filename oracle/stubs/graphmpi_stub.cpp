// Test-harness shim: a no-op Graphmpi so the reference CPU sources link
// without MPI.  Only Graph::pattern_matching_mpi (reference src/graph.cpp:568)
// names Graphmpi and the oracle binaries never reach it.  Test
// infrastructure only; not part of the engine.
#include "graphmpi.h"

Graphmpi &Graphmpi::getinstance() {
    static Graphmpi only;
    return only;
}
std::pair<int, int> Graphmpi::init(int, Graph *) { return std::make_pair(-1, -1); }
long long Graphmpi::runmajor() { return 0; }
int *Graphmpi::getneighbor(int) { return nullptr; }
int Graphmpi::getdegree() { return 0; }
bool Graphmpi::include(int) { return true; }
std::pair<int, int> Graphmpi::get_vertex_range() { return std::make_pair(-1, -1); }
void Graphmpi::report(long long) {}
void Graphmpi::end() {}
Graphmpi::Graphmpi() {}
Graphmpi::~Graphmpi() {}
