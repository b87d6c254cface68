// svdag_replay.cu - the reference's recorded edit sessions (ReplayManager::load_csv, replay.h:650-690)
// as requests: one action per line, the action name then comma-separated values. Positions and radii
// are scaled from the replay's grid to the scene's (scalingFactor, replay.cpp:10), exactly as the
// reference's ReplayAction*::apply (replay.cpp:52-134) passes them to the MyGpu editors.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/svdag.h"

namespace {

// std::stof / std::stoi as the reference's loaders use them (whole leading number; the rest ignored).
bool to_float(const std::string& s, float& out)
{
    const char* b = s.c_str();
    char* e = nullptr;
    out = std::strtof(b, &e);
    return e != b;
}
bool to_int(const std::string& s, long& out)
{
    const char* b = s.c_str();
    char* e = nullptr;
    out = std::strtol(b, &e, 10);
    return e != b;
}
bool to_bool(const std::string& s, bool& out)
{
    if (s == "true" || s == "TRUE") {
        out = true;
        return true;
    }
    if (s == "false" || s == "FALSE") {
        out = false;
        return true;
    }
    return false;
}

// One line: the action name and its cells (trailing empty cells removed, as load_csv does).
bool parse_action(const std::string& name, const std::vector<std::string>& d, float scale, svdag_replay_action& a)
{
    std::memset(&a, 0, sizeof(a));
    a.kind = SVDAG_REPLAY_OTHER;
    auto vec3 = [&](size_t at, float* v) {
        for (int i = 0; i < 3; ++i)
            if (!to_float(d[at + i], v[i]))
                return false;
        return true;
    };
    if (name == "EndFrame") {
        a.kind = SVDAG_REPLAY_END_FRAME;
        return true;
    }
    if (name == "Undo" || name == "Redo") {
        a.kind = name == "Undo" ? SVDAG_REPLAY_UNDO : SVDAG_REPLAY_REDO;
        return true;
    }
    if (name == "SetLocation" || name == "SetRotation") {
        const size_t n = name == "SetLocation" ? 3 : 9;
        if (d.size() != n)
            return false;
        a.kind = n == 3 ? SVDAG_REPLAY_CAMERA_LOCATION : SVDAG_REPLAY_CAMERA_ROTATION;
        for (size_t i = 0; i < n; ++i) {
            float v;
            if (!to_float(d[i], v))
                return false;
            a.camera[i] = v;
        }
        return true;
    }
    auto numbers = [&](size_t from, size_t to) {
        for (size_t i = from; i < to; ++i) {
            float v;
            if (!to_float(d[i], v))
                return false;
        }
        return true;
    };
    if (name == "SetToolParameters") // the interactive tool's cursor state (replay.h:246-265): no edit of its own
        return (d.size() == 11 || d.size() == 14) && numbers(0, d.size());
    if (name == "EditFill") // FillEditorColors edits the CPU HashDAG only
        return d.size() == 4 && numbers(0, 4);
    svdag_edit& e = a.edit;
    float loc[3], radius;
    if (name == "EditSphere" || name == "EditCube") { // ReplayActionSphere/Cube::load, replay.h:288-376
        bool add;
        long mat = 1;
        if ((d.size() != 5 && d.size() != 6) || !vec3(0, loc) || !to_float(d[3], radius) || !to_bool(d[4], add)
            || (d.size() > 5 && !to_int(d[5], mat)))
            return false;
        const bool sphere = name == "EditSphere";
        e.tool = sphere ? (add ? SVDAG_TOOL_SPHERE_ADD : SVDAG_TOOL_SPHERE_REMOVE) : (add ? SVDAG_TOOL_BOX_ADD : SVDAG_TOOL_BOX_REMOVE);
        e.material = (uint32_t)mat;
    } else if (name == "EditPaint") { // ReplayActionPaint::load, replay.h:495-541 (the colour is not stored in the DAG)
        long mat = 1;
        if ((d.size() != 4 && d.size() != 7 && d.size() != 8) || !vec3(0, loc) || !to_float(d[3], radius)
            || (d.size() > 7 && !to_int(d[7], mat)))
            return false;
        e.tool = SVDAG_TOOL_SPHERE_PAINT;
        e.material = (uint32_t)mat;
    } else if (name == "EditCopy") { // ReplayActionCopy::load, replay.h:378-458 (MyGpuCopyEditor ignores transform and swirl)
        float src[3], dst[3];
        bool swirl;
        if ((d.size() != 10 && d.size() != 21) || !vec3(0, loc) || !vec3(3, src) || !vec3(6, dst) || !to_float(d[9], radius)
            || (d.size() == 21 && (!numbers(10, 19) || !to_bool(d[19], swirl) || !numbers(20, 21))))
            return false;
        e.tool = SVDAG_TOOL_COPY;
        for (int i = 0; i < 3; ++i) {
            e.src[i] = src[i] * scale;
            e.dst[i] = dst[i] * scale;
        }
    } else {
        return false;
    }
    if (e.material >= SVDAG_NUM_MATERIALS)
        return false;
    for (int i = 0; i < 3; ++i)
        e.center[i] = loc[i] * scale;
    e.radius = radius * scale;
    a.kind = SVDAG_REPLAY_EDIT;
    return true;
}

} // namespace

extern "C" svdag_status svdag_replay_parse(const char* text, uint64_t length, float scale, svdag_replay_action* out, uint64_t capacity,
    uint64_t* count, uint64_t* badLine)
{
    if (!count || (length && !text) || (capacity && !out) || !(scale > 0.0f))
        return SVDAG_ERR_INVALID;
    uint64_t n = 0, line = 0;
    std::vector<std::string> cells;
    auto finish = [&]() -> bool {
        if (!cells.empty() && !cells.back().empty() && cells.back().back() == '\r') // CRLF files
            cells.back().pop_back();
        if (cells.empty() || (cells.size() == 1 && cells[0].empty()))
            return true; // blank line
        const std::string name = cells.front();
        cells.erase(cells.begin());
        while (!cells.empty() && cells.back().empty())
            cells.pop_back();
        svdag_replay_action a;
        if (!parse_action(name, cells, scale, a))
            return false;
        if (n < capacity)
            out[n] = a;
        ++n;
        cells.clear();
        return true;
    };
    for (uint64_t i = 0; i < length; ++i) {
        const char c = text[i];
        if (c == '\n') {
            if (!finish()) {
                if (badLine)
                    *badLine = line;
                *count = n;
                return SVDAG_ERR_INVALID;
            }
            cells.clear();
            ++line;
        } else if (c == ',') {
            cells.emplace_back();
        } else {
            if (cells.empty())
                cells.emplace_back();
            cells.back().push_back(c);
        }
    }
    // Text after the last newline is not an action: load_csv only completes a line at '\n'.
    *count = n;
    return n > capacity && capacity ? SVDAG_ERR_OOM : SVDAG_OK;
}
