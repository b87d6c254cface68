// Host build of the serving loop's geometry (gpu-svdag-editing_b200/csrc/svdag_serve_geometry.h) for
// the CPU tests: the same edit_reserve_bytes, edit_boxes and box_rows the server runs. Test
// infrastructure only.
#include "../gpu-svdag-editing_b200/csrc/svdag_serve_geometry.h"

extern "C" {

uint32_t frames_edit_boxes(const svdag_edit* e, float* out) { return svdag::serve::edit_boxes(*e, out); }

// rows and columns as out[0..3] = row0, row1, col0, col1; returns 0 when the box is not wholly in front
int frames_box_rows(const svdag_trace_params* p, const float* box, int64_t* out)
{
    return svdag::serve::box_rows(*p, box, out[0], out[1], out[2], out[3]) ? 1 : 0;
}

unsigned long long frames_edit_reserve_bytes(const svdag_edit* e, uint32_t levels)
{
    return svdag::serve::edit_reserve_bytes(*e, levels);
}

} // extern "C"
