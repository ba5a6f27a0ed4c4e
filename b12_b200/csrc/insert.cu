// Insertion of new boxes (continuation).  Filled in with the radix sort.
#include "tree.h"

using namespace b12g::host;

extern "C" {

b12g_status b12g_insert_points(b12g_tree* t, const double*, uint64_t, uint8_t, uint8_t, uint8_t, uint32_t*)
{
  return fail(B12G_ERR_INVALID, "insert_points: not built yet");
}

b12g_status b12g_insert_by_image(b12g_tree* t, const b12g_scheme*, uint8_t, uint8_t, uint8_t, uint32_t*)
{
  return fail(B12G_ERR_INVALID, "insert_by_image: not built yet");
}

b12g_status b12g_continuation_run(b12g_tree*, const b12g_scheme*, const double*, uint64_t, uint8_t, uint32_t,
                                  uint32_t*, uint32_t*)
{
  return fail(B12G_ERR_INVALID, "continuation_run: not built yet");
}

}
