// cudaSortedPositions (cudaSortedPositions.hh:6-36): the sorted copy of the
// positions is built with the cell list inside the library.
#if !defined(CUDASORTEDPOSITIONS)
#define CUDASORTEDPOSITIONS

#include "cudaParticleBase.hh"

class cudaSortedPositions : public virtual cudaParticleBase {
 public:
  void reset(void) {}
};

#endif /* CUDASORTEDPOSITIONS */
