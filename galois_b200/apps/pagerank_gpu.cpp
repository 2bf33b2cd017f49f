// pagerank-gpu: the pull app, lonestar/analytics/cpu/pagerank/PageRank-pull.cpp
// (-algo=Residual, the default, or Topo) on the device; see pagerank_app.h.
#include "pagerank_app.h"

int main(int argc, char** argv) { return pagerank_app(argc, argv, false); }
