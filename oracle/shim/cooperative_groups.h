/* Host-only stand-in for <cooperative_groups.h>: the reference's hashers name
 * cg::thread_block_tile<N> in a device-only overload that the pin never calls. */
#pragma once
#include <cstddef>
namespace cooperative_groups {
template <unsigned int N, typename P = void>
class thread_block_tile {};
}
