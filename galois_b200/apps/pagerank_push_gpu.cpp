// pagerank-push-gpu: the push app, lonestar/analytics/cpu/pagerank/
// PageRank-push.cpp (-algo=Async, the default, or Sync) on the device; see
// pagerank_app.h.
#include "pagerank_app.h"

int main(int argc, char** argv) { return pagerank_app(argc, argv, true); }
