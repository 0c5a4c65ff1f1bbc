// Host particle record with the reference's field names and byte layout
// (ParticleBase.hh:10-18); pb_particle in pb/pb.h is the same record.
#if !defined(PARTICLEBASE)
#define PARTICLEBASE

#include <cstdint>

class ParticleBase {
 public:
  double r[3];
  double m;
  double v[3];
  bool isFixed;
  double a[3];
  uint32_t type;
};

#endif
