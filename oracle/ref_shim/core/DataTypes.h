// Minimal stand-in for waLBerla's core/DataTypes.h (submodule absent): the scalar type names the
// reference's generated kernels use.  Test infrastructure only.
#pragma once
#include <cstddef>
#include <cstdint>
namespace walberla {
using float64 = double;
using float32 = float;
using real_t  = double;
using uint_t  = std::size_t;
template < typename T >
inline real_t real_c( T t )
{
   return real_t( t );
}
}  // namespace walberla
