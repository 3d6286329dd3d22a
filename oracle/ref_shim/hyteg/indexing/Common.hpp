// Minimal stand-in for hyteg/indexing/Common.hpp: a 3-component logical index ordered z-major, as
// the reference orders it (src/hyteg/indexing/Common.hpp:67-71).  Test infrastructure only.
#pragma once
#include <cstdint>
namespace hyteg {
using idx_t = std::int64_t;
namespace indexing {
class Index
{
 public:
   Index() = default;
   Index( idx_t x, idx_t y, idx_t z )
   : v_{ x, y, z }
   {}
   idx_t x() const { return v_[0]; }
   idx_t y() const { return v_[1]; }
   idx_t z() const { return v_[2]; }

 private:
   idx_t v_[3] = { 0, 0, 0 };
};
inline bool operator<( const Index& a, const Index& b )
{
   return a.z() < b.z() || ( a.z() == b.z() && a.y() < b.y() ) || ( a.z() == b.z() && a.y() == b.y() && a.x() < b.x() );
}
}  // namespace indexing
}  // namespace hyteg
