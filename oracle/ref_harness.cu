// ref_harness.cu - the reference's own host-callable code behind a C API, to check the oracle.
//
// TEST INFRASTRUCTURE ONLY (like the rest of oracle/): tests compare the oracle and the CUDA
// library against these functions; nothing in the product loads the built library. It is compiled
// by oracle/build_ref.py from the reference sources where they lie (nothing is copied), with the
// stand-ins of oracle/ref_shim for the two external libraries the headers include (gsl-lite's span
// and narrow, TBB's parallel_for_each), into oracle/_ref/libref.so.
//
// What runs here is the reference's code, called from the host:
//  - the editors (my_gpu_dag_editors.h): MyGpuSphereEditor<isAdding> (:457-496), MyGpuBoxEditor
//    (:82-119), MyGpuSpherePaintEditor (:498-536), MyGpuCopyEditor (:127-253, the stateful form)
//    and MyGpuSphereErosionEditor (:538-589), their should_edit and get_new_value;
//  - GPUBaseDAG (my_gpu_base_dag.h:86-351): LeafBuilder_, the node header codecs,
//    get_node_is_fully_filled, get_material, get_leaf_size;
//  - DAGUtils::get_value (dag_utils.h:146-182) and Path (path.h).
// The DAG they read is RefDag below: items at a stride of 10 words with children given as item
// indices (an export of the oracle's or the CUDA library's DAG), with the reference's item encoding.
//
// ref_edit_values evaluates an edit per voxel the way createIntermediateSvoStructure decides it
// (create_edit_svo.cu:167-303 for the inner levels, :321-426 for the leaf voxels, with
// FILL_FULL_REGION and EDITS_ENABLE_MATERIALS set as the reference's configuration sets them): from
// the root, each child's NodeDesc from the DAG before the edit, the editor's should_edit, Keep /
// Empty / Fill ending the descent, Subdivide continuing it; at the leaf, should_edit of the voxel
// and get_new_value. The traversal is this file's; every decision and value is the reference
// editor's.
#include "configuration/script_definitions.h"
#include "typedefs.h"

#include "dags/dag_utils.h"
#include "dags/my_gpu_dags/my_gpu_base_dag.h"
#include "dags/my_gpu_dags/my_gpu_dag_editors.h"
#include "path.h"

#include <cstdint>
#include <optional>
#include <vector>

#include "../include/svdag.h"

namespace {

constexpr uint32_t kNoValue = 0xFFFFFFFFu; // an empty voxel / a missing child

struct RefDag : GPUBaseDAG<RefDag, HASH_DAG_MATERIAL_BITS> {
    const uint32_t* items = nullptr; // 10 words per item
    uint32_t levels = 0; // hides BaseDAG::levels (the reference's compile-time depth)
    uint32_t root = kNoValue;

    HOST_DEVICE uint32_t leaf_level() const { return levels - 2; }
    HOST_DEVICE uint32_t get_first_node_index() const { return root; }
    HOST_DEVICE const uint32_t* get_node_ptr(uint32_t, uint32_t handle) const { return items + 10ull * handle; }
    HOST_DEVICE const uint32_t* get_leaf_ptr(uint32_t handle) const { return items + 10ull * handle; }
};

struct Holder {
    std::vector<uint32_t> words;
    RefDag dag;
};

float3 f3(const float* v) { return make_float3(v[0], v[1], v[2]); }

uint32_t old_value(const RefDag& dag, uint32_t x, uint32_t y, uint32_t z)
{
    if (dag.root == kNoValue)
        return kNoValue;
    const std::optional<uint32_t> v = DAGUtils::get_value(dag, Path(x, y, z));
    return v ? *v : kNoValue;
}

template <typename Editor>
constexpr bool kStateful = requires(const Editor& e) { e.createInitialState(); };

template <typename Editor>
uint32_t edit_voxel(const RefDag& dag, const Editor& editor, uint32_t x, uint32_t y, uint32_t z)
{
    uint32_t handle = dag.root;
    Path path(0, 0, 0);
    const Path voxel(x, y, z);
    const uint32_t L = dag.levels;
    auto state = [&] {
        if constexpr (kStateful<Editor>)
            return editor.createInitialState();
        else
            return 0;
    }();
    for (uint32_t level = 0; level < dag.leaf_level(); ++level) {
        const uint8_t c = voxel.child_index(level + 1, L);
        uint32_t child = kNoValue;
        if (handle != kNoValue) {
            const uint32_t* node = dag.get_node_ptr(level, handle);
            const uint8_t mask = Utils::child_mask(node[0]);
            if (mask & (1u << c))
                child = dag.get_child_index(level, node, mask, c);
        }
        Path childPath = path;
        childPath.descend(c);
        const uint32_t childLevel = level + 1;
        const uint32_t childDepth = L - childLevel;
        NodeDesc desc {};
        desc.fillMaterial = 0;
        if (child == kNoValue)
            desc.state = NodeState::Empty;
        else if (childLevel == dag.leaf_level())
            desc.state = NodeState::Partial;
        else
            desc.state = RefDag::get_node_is_fully_filled(dag.get_node_ptr(childLevel, child)[0], desc.fillMaterial) ? NodeState::Filled
                                                                                                                  : NodeState::Partial;
        NodeEditDesc d;
        if constexpr (kStateful<Editor>) {
            decltype(state) next {};
            d = editor.should_edit(childPath, childDepth, desc, state, next);
            state = next;
        } else {
            d = editor.should_edit(childPath, childDepth, desc);
        }
        if (d.operation == EditOperation::Keep)
            return old_value(dag, x, y, z);
        if (d.operation == EditOperation::Empty)
            return kNoValue;
        if (d.operation == EditOperation::Fill)
            return d.fillMaterial;
        handle = child;
        path = childPath;
    }
    const uint32_t v = ((x & 1u) ? 4u : 0u) | ((y & 1u) ? 2u : 0u) | ((z & 1u) ? 1u : 0u) | ((x & 2u) ? 32u : 0u) | ((y & 2u) ? 16u : 0u)
        | ((z & 2u) ? 8u : 0u);
    std::optional<uint32_t> old;
    if (handle != kNoValue) {
        uint32_t m;
        if (RefDag::get_material(dag.get_leaf_ptr(handle), v, m))
            old = m;
    }
    Path vp = path;
    vp.descend(uint8_t(v >> 3));
    vp.descend(uint8_t(v & 7u));
    NodeDesc desc {};
    if (old) {
        desc.state = NodeState::Filled;
        desc.fillMaterial = *old;
    } else {
        desc.state = NodeState::Empty;
        desc.fillMaterial = 0xFFFFFFFFu;
    }
    const NodeEditDesc d = editor.should_edit(vp, 0, desc);
    std::optional<uint32_t> out;
    if (d.operation == EditOperation::Fill || d.operation == EditOperation::Subdivide) {
        if constexpr (kStateful<Editor>)
            out = editor.get_new_value(vp.path, old, state);
        else
            out = editor.get_new_value(vp.as_position(0), old);
    } else if (d.operation == EditOperation::Keep) {
        out = old;
    }
    return out ? *out : kNoValue;
}

template <typename Editor>
void edit_all(const RefDag& dag, const Editor& editor, const uint32_t* xyz, uint64_t n, uint32_t* out)
{
    for (uint64_t i = 0; i < n; ++i)
        out[i] = edit_voxel(dag, editor, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}

// Calls `f` with the reference editor of the edit; false for a tool the reference does not have.
template <typename F>
bool with_editor(const svdag_edit& e, const RefDag& dag, F&& f)
{
    switch (e.tool) {
    case SVDAG_TOOL_SPHERE_ADD:
        f(MyGpuSphereEditor<true>(f3(e.center), e.radius, e.material));
        return true;
    case SVDAG_TOOL_SPHERE_REMOVE:
        f(MyGpuSphereEditor<false>(f3(e.center), e.radius, e.material));
        return true;
    case SVDAG_TOOL_BOX_ADD:
        f(MyGpuBoxEditor<true>(f3(e.center), e.radius, e.material));
        return true;
    case SVDAG_TOOL_BOX_REMOVE:
        f(MyGpuBoxEditor<false>(f3(e.center), e.radius, e.material));
        return true;
    case SVDAG_TOOL_SPHERE_PAINT:
        f(MyGpuSpherePaintEditor(f3(e.center), e.radius, make_float3(0.0f), e.material));
        return true;
    case SVDAG_TOOL_COPY:
        f(MyGpuCopyEditor<RefDag>(dag, f3(e.src), f3(e.dst), f3(e.center), e.radius));
        return true;
    case SVDAG_TOOL_SPHERE_ERODE:
        f(MyGpuSphereErosionEditor<RefDag>(dag, f3(e.center), e.radius, e.noise_seed));
        return true;
    default:
        return false;
    }
}

using Leaf4 = GPUBaseDAG<RefDag, HASH_DAG_MATERIAL_BITS>;

} // namespace

extern "C" {

void* ref_dag_create(uint32_t levels, const uint32_t* items, uint64_t count)
{
    auto* h = new Holder();
    h->words.assign(items, items + 10ull * count);
    h->dag.items = h->words.data();
    h->dag.levels = levels;
    h->dag.root = count ? 0u : kNoValue;
    return h;
}

void ref_dag_destroy(void* h) { delete static_cast<Holder*>(h); }

// DAGUtils::get_value for each voxel: its material, or 0xFFFFFFFF for an empty voxel.
int ref_get_values(const void* h, const uint32_t* xyz, uint64_t n, uint32_t* out)
{
    const RefDag& dag = static_cast<const Holder*>(h)->dag;
    for (uint64_t i = 0; i < n; ++i)
        out[i] = old_value(dag, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    return 0;
}

// The voxels' values after the edit, evaluated from the DAG before it; 1 for a tool the reference
// does not have (the procedural noise paint).
int ref_edit_values(const void* h, const svdag_edit* e, const uint32_t* xyz, uint64_t n, uint32_t* out)
{
    const RefDag& dag = static_cast<const Holder*>(h)->dag;
    return with_editor(*e, dag, [&](const auto& editor) { edit_all(dag, editor, xyz, n, out); }) ? 0 : 1;
}

// The editor's decision for one node (the stateless should_edit; the copy editor's stateless form
// is its overlap test). Returns the EditOperation (0 Subdivide, 1 Fill, 2 Empty, 3 Keep), or -1 for
// a tool the reference does not have.
int ref_should_edit(const svdag_edit* e, const uint32_t path[3], uint32_t depth, uint32_t state, uint32_t fill, uint32_t* out_fill)
{
    RefDag empty;
    empty.levels = SVDAG_MAX_LEVELS;
    const Path p(path[0], path[1], path[2]);
    NodeDesc desc {};
    desc.state = state == 0 ? NodeState::Partial : (state == 1 ? NodeState::Filled : NodeState::Empty);
    desc.fillMaterial = fill;
    int op = -1;
    with_editor(*e, empty, [&](const auto& editor) {
        const NodeEditDesc d = editor.should_edit(p, depth, desc);
        op = (int)d.operation;
        if (out_fill)
            *out_fill = d.fillMaterial;
    });
    return op;
}

// ref_should_edit over n nodes of one edit: paths (3 words each), depths, states and fill
// materials in; operations and fill materials out.
int ref_should_edit_many(const svdag_edit* e, const uint32_t* paths, const uint32_t* depths, const uint32_t* states,
    const uint32_t* fills, uint64_t n, int32_t* ops, uint32_t* outFills)
{
    for (uint64_t i = 0; i < n; ++i) {
        ops[i] = ref_should_edit(e, paths + 3 * i, depths[i], states[i], fills[i], outFills + i);
        if (ops[i] < 0)
            return 1;
    }
    return 0;
}

// LeafBuilder_ over 64 voxels in voxel-index order (0xFFFFFFFF = empty); returns the leaf size.
uint32_t ref_build_leaf(const uint32_t* materials, uint32_t* out)
{
    Leaf4::LeafBuilder_ b(out);
    for (uint32_t v = 0; v < 64; ++v) {
        if (materials[v] != kNoValue)
            b.set(materials[v]);
        b.next();
    }
    return b.finalize();
}

uint32_t ref_leaf_size(const uint32_t* leaf) { return Leaf4::get_leaf_size(leaf); }
int ref_leaf_material(const uint32_t* leaf, uint32_t voxel, uint32_t* out) { return Leaf4::get_material(leaf, voxel, *out) ? 1 : 0; }

uint32_t ref_encode_node_header(uint32_t child_mask, uint32_t user_payload)
{
    uint32_t w = 0;
    Leaf4::encode_node_header_with_payload(&w, child_mask, user_payload);
    return w;
}
uint32_t ref_encode_full_node_header(uint32_t child_mask, uint32_t material)
{
    uint32_t w = 0;
    Leaf4::encode_node_header(&w, child_mask, material);
    return w;
}
// get_node_is_fully_filled: 1 and the material when the header carries the flag.
int ref_header_fully_filled(uint32_t header, uint32_t* material) { return Leaf4::get_node_is_fully_filled(header, *material) ? 1 : 0; }

} // extern "C"
