/* Declaration of the one arbok class the reference's cbm/cbm_extensions.cpp
 * names (arbok::TarjanPQ, used by cbm_init_ at :154-189) -- TEST
 * INFRASTRUCTURE ONLY (oracle/build_ref.py).
 *
 * arbok (github.com/chistopher/arbok) is an absent, unpinned submodule of the
 * reference.  This header only lets the reference's source file compile so
 * that its eight product operators can be built and timed; it declares the
 * members cbm_init_ calls and defines none of them.  The built module is
 * loaded with lazy symbol binding and its init is never called: a call would
 * stop at the first unresolved symbol. */
#ifndef CBM_REF_SHIM_ARBOK_TARJAN_PQ_H
#define CBM_REF_SHIM_ARBOK_TARJAN_PQ_H

#include <vector>

namespace arbok {
class TarjanPQ {
 public:
  TarjanPQ(int n, int m);
  ~TarjanPQ();
  void create_edge(int from, int to, long long weight);
  long long run(int root);
  std::vector<int> reconstruct(int root);
};
}  // namespace arbok
#endif
