# RadiativeViewFactorB200Ext -- the package extension that plugs librvf_b200
# into RadiativeViewFactor.jl's GPU hook (src/Assembly.jl:241-260).
#
# It defines a backend type with the registry methods the reference's
# extensions add (ext/RadiativeViewFactorCUDAExt.jl:11-12), wraps the hook
# already registered (compute_view_factors_gpu, src/GPUAssembly.jl:111) so
# that every other backend keeps its own path, flattens MeshData with the
# reference's own build_gpu_arrays (src/GPUKernels.jl:336-412) and calls the
# C ABI of include/rvf_b200.h through ccall.  With the companion patch
# julia/patches/Assembly_gpu_supports.diff applied, the trait
# _gpu_supports(backend, feature) lets compute_view_factors pass use_duffy,
# self_vf, seed and curve meshes (mesh_dim == 1) through to this backend.
#
# The structs below mirror rvf_mesh_desc, rvf_options, rvf_stats,
# rvf_server_opts and rvf_request_info field for field; a test of this
# repository parses them and checks every offset against the compiled header.
#
# This file cannot be executed where it was written (no Julia toolchain):
# the same C ABI is exercised from Python through ctypes by the test-suite.
module RadiativeViewFactorB200Ext

using RadiativeViewFactor
import RadiativeViewFactor.Assembly: _gpu_array_type, _gpu_float_type, _gpu_supports, _GPU_HOOK_REF,
                                     register_gpu_hook!
import RadiativeViewFactor.GPUKernels: build_gpu_arrays
import RadiativeViewFactor.Results: ViewFactorResult

const LIB = get(ENV, "RVF_B200_LIB", "librvf_b200.so")

struct B200Backend end
_gpu_array_type(::B200Backend) = Array     # host arrays: the library owns device memory
_gpu_float_type(::B200Backend) = Float64
_gpu_supports(::B200Backend, feature::Symbol) = feature in (:duffy, :curves, :self_vf, :seed)

struct RvfMeshDesc
    mesh_dim::Int32
    n_nodes::Int64
    coords::Ptr{Float64}
    n_elems::Int64
    elem_family::Ptr{Int8}
    elem_node_idx::Ptr{Int32}
    elem_group::Ptr{Int32}
    nodes::NTuple{6,Ptr{Int32}}
    n_family::NTuple{6,Int64}
    n_obs::Int64
    obs_nv::Int32
    obs_soup::Ptr{Float64}
    obs_group::Ptr{Int32}
    n_groups::Int32
    group_tags::Ptr{Int32}
end

struct RvfOptions
    nquad::Int32
    method::Int32
    use_duffy::Int32
    n_samples::Int32
    seed::UInt64
    precision::Int32
    occlusion::Int32
    geometric_soup::Int32
    mc_exclude_groups::Int32
    near_field_factor::Float64
    ray_log::Ptr{UInt8}
    ray_log_pm::Int32
    disable_pair_lists::Int32
    self_vf::Int32
    disable_tile_cull::Int32
    fault_inject::Int32
    fast_points::Int32
    fast_row_groups::Int32
    reserved::NTuple{2,Int32}
end

struct RvfStats
    ms_upload::Float64
    ms_prep::Float64
    ms_pairs::Float64
    ms_duffy::Float64
    ms_reduce::Float64
    ms_download::Float64
    ms_total::Float64
    n_pairs::Int64
    n_point_pairs::Int64
    n_rays::Int64
    n_rays_fp64::Int64
    n_pairs_fp64::Int64
    n_duffy_pairs::Int64
    max_row_sum_dev::Float64
    n_node_visits::Int64
    n_prim_tests::Int64
    n_kernels::Int64
    n_graze_fp64::Int64
    n_unsure_rays::Int64
    n_unsure_slab::Int64
    n_unsure_prim::Int64
    n_unsure_dir::Int64
    n_rays_traced::Int64
    n_chunks::Int64
    ms_gen::Float64
    ms_trace::Float64
    ms_trace_fp64::Float64
    ms_resolve::Float64
    n_list_pairs::Int64
    n_walk_pairs::Int64
    ms_lists::Float64
    n_tiles_culled::Int64
    n_pairs_masked::Int64
    ms_cull::Float64
    n_tiles_unclassified::Int64
    reserved::NTuple{1,Int64}
end

struct RvfServerOpts
    admit_bytes::UInt64
    max_batch::Int32
    use_graphs::Int32
    autotune::Int32
    reserved::NTuple{8,Int32}
end

struct RvfRequestInfo
    state::Int32
    status::Int32
    n_elems::Int64
    footprint_bytes::UInt64
    t_submit_ms::Float64
    t_admit_ms::Float64
    t_done_ms::Float64
    n_chunks::Int64
    reserved::NTuple{8,Int32}
end

struct RvfTunedShape
    mixed::Int32
    occlusion::Int32
    dim3::Int32
    size_class::Int32
    gen_blocks_per_sm::Int32
    trace_blocks_per_sm::Int32
    fast_points::Int32
    fast_row_groups::Int32
    rule_points::Int32
    reserved::Int32
    fast_ms_per_gpp::Float64
    fast_ms_per_gpp_default::Float64
end

struct RvfServerStats
    submitted::Int64
    completed::Int64
    failed::Int64
    canceled::Int64
    in_flight::Int64
    p50_ms::Float64
    p99_ms::Float64
    mean_ms::Float64
    wall_ms::Float64
    pairs_done::Int64
    chunks::Int64
    graph_replays::Int64
    batched_requests::Int64
    admitted_bytes_peak::UInt64
    n_tuned::Int32
    reserved::Int32
    ms_admit::Float64
    ms_quad_chunks::Float64
    ms_mc_chunks::Float64
    ms_free::Float64
    ms_idle::Float64
    tuned::NTuple{8,RvfTunedShape}
end

const RVF_PREC_FP64 = Int32(0)
const RVF_PREC_MIXED = Int32(1)

const SESSION = Ref{Ptr{Cvoid}}(C_NULL)

function check(rc)
    rc == 0 && return
    buf = Vector{UInt8}(undef, 4096)
    ccall((:rvf_last_error, LIB), Cint, (Ptr{UInt8}, Csize_t), buf, length(buf))
    error(unsafe_string(pointer(buf)))
end

function session()
    if SESSION[] == C_NULL
        out = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:rvf_session_create, LIB), Cint, (Ptr{Cvoid}, Ref{Ptr{Cvoid}}), C_NULL, out))
        SESSION[] = out[]
    end
    SESSION[]
end

function default_options()
    o = Ref{RvfOptions}()
    ccall((:rvf_default_options, LIB), Cvoid, (Ref{RvfOptions},), o)
    o[]
end

# a copy of `o` with some fields replaced
function with(o::RvfOptions; kw...)
    vals = [haskey(kw, f) ? convert(fieldtype(RvfOptions, f), kw[f]) : getfield(o, f)
            for f in fieldnames(RvfOptions)]
    RvfOptions(vals...)
end

# The merged obstruction soup in obstruction_groups order with per-triangle
# group tags (what build_flat_bvh_from_mesh merges, src/GPUBVH.jl:146-174).
function merged_soup(mesh, obstruction_groups)
    groups = [g for g in obstruction_groups if haskey(mesh.group_tri_soup, g)]
    nv = mesh.mesh_dim == 1 ? 2 : 3
    isempty(groups) && return zeros(3, nv, 0), Int32[]
    soup = cat((mesh.group_tri_soup[g] for g in groups)...; dims=3)
    tags = reduce(vcat, [fill(Int32(g), size(mesh.group_tri_soup[g], 3)) for g in groups])
    soup, tags
end

function compute_view_factors_b200(mesh, nquad, backend, FloatT, ArrayT;
                                   obstruction_groups=Int[], verbose=true,
                                   monte_carlo=false, n_samples=10000,
                                   use_duffy=false, self_vf=false, seed=rand(UInt64),
                                   precision=RVF_PREC_FP64)
    ga = build_gpu_arrays(mesh, nquad, Array, Float64)    # the reference's own flattening
    soup, tags = merged_soup(mesh, obstruction_groups)
    gtags = Int32.(sort(collect(keys(mesh.group_tags))))
    N, G = length(mesh.surface_elems), length(gtags)
    empty = Int32[]
    tbl(x) = isempty(x) ? pointer(empty) : pointer(x)
    verbose && println("B200 compute_view_factors: $N elements, nquad=$nquad")
    GC.@preserve ga soup tags gtags empty begin
        d = RvfMeshDesc(mesh.mesh_dim, size(ga.coords, 2), pointer(ga.coords), N,
                        pointer(ga.elem_family), pointer(ga.elem_node_idx), pointer(ga.elem_group),
                        (tbl(ga.nodes_quad), tbl(ga.nodes_tri), tbl(ga.nodes_quad4), tbl(ga.nodes_tri3),
                         Ptr{Int32}(C_NULL), Ptr{Int32}(C_NULL)),
                        (size(ga.nodes_quad, 2), size(ga.nodes_tri, 2), size(ga.nodes_quad4, 2),
                         size(ga.nodes_tri3, 2), 0, 0),
                        size(soup, 3), size(soup, 2), pointer(soup), tbl(tags), G, pointer(gtags))
        m = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:rvf_mesh_upload, LIB), Cint, (Ptr{Cvoid}, Ref{RvfMeshDesc}, Ref{Ptr{Cvoid}}),
                    session(), d, m))
        F, A = Matrix{Float64}(undef, N, N), Vector{Float64}(undef, N)
        Fg, Ag = Matrix{Float64}(undef, G, G), Vector{Float64}(undef, G)
        o = with(default_options(); nquad=nquad, method=monte_carlo ? 1 : 0, use_duffy=use_duffy,
                 n_samples=n_samples, seed=seed, precision=precision, self_vf=self_vf)
        st = Ref{RvfStats}()
        try
            check(ccall((:rvf_solve, LIB), Cint,
                        (Ptr{Cvoid}, Ptr{Cvoid}, Ref{RvfOptions}, Ptr{Float64}, Ptr{Float64},
                         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ref{RvfStats}),
                        session(), m[], o, F, A, Fg, Ag, C_NULL, st))
        finally
            ccall((:rvf_mesh_release, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), session(), m[])
        end
        verbose && println("  pairs $(st[].n_pairs), rays $(st[].n_rays), $(round(st[].ms_total; digits=1)) ms")
        names = [mesh.group_tags[t] for t in gtags]
        return ViewFactorResult(F, A, Fg, Ag, Int.(gtags), names)
    end
end

function __init__()
    previous = _GPU_HOOK_REF[]                  # compute_view_factors_gpu, registered at load
    register_gpu_hook!((mesh, nquad, backend, FloatT, ArrayT; kw...) ->
        backend isa B200Backend ?
            compute_view_factors_b200(mesh, nquad, backend, FloatT, ArrayT; kw...) :
            previous(mesh, nquad, backend, FloatT, ArrayT; kw...))
end

# ---------------------------------------------------------------------------
# Request loop (serving): one server per GPU, solves submitted as they arrive
# and collected out of order; the library batches admitted requests.
# ---------------------------------------------------------------------------
function server(; admit_bytes=0)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    o = RvfServerOpts(admit_bytes, 0, 0, 0, ntuple(_ -> Int32(0), 8))
    check(ccall((:rvf_server_create, LIB), Cint, (Ptr{Cvoid}, Ref{RvfServerOpts}, Ref{Ptr{Cvoid}}),
                session(), o, out))
    out[]
end

# d and o are built as in compute_view_factors_b200 (the arrays behind d must
# stay alive until submit returns: the library copies them)
function submit(sv, d::RvfMeshDesc, o::RvfOptions)
    id = Ref{Int64}(0)
    check(ccall((:rvf_submit, LIB), Cint, (Ptr{Cvoid}, Ref{RvfMeshDesc}, Ref{RvfOptions}, Ref{Int64}),
                sv, d, o, id))
    id[]
end

# blocks until request `id` is done, copies its result and releases it
function collect!(sv, id, N, G)
    info = Ref{RvfRequestInfo}()
    check(ccall((:rvf_wait, LIB), Cint, (Ptr{Cvoid}, Int64, Int64, Ref{RvfRequestInfo}), sv, id, -1, info))
    F, A = Matrix{Float64}(undef, N, N), Vector{Float64}(undef, N)
    Fg, Ag = Matrix{Float64}(undef, G, G), Vector{Float64}(undef, G)
    check(ccall((:rvf_request_result, LIB), Cint,
                (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                sv, id, F, A, Fg, Ag, C_NULL))
    check(ccall((:rvf_release, LIB), Cint, (Ptr{Cvoid}, Int64), sv, id))
    F, A, Fg, Ag
end

# the id of the next request to finish (in finishing order), or nothing at the time limit
function wait_any(sv; timeout_ms=-1)
    id = Ref{Int64}(0)
    rc = ccall((:rvf_wait_any, LIB), Cint, (Ptr{Cvoid}, Int64, Ref{Int64}), sv, timeout_ms, id)
    rc == -5 && return nothing  # RVF_ETIMEDOUT
    check(rc)
    id[]
end

# counts, latency percentiles and the autotuner's chosen launch shapes
function stats(sv)
    st = Ref{RvfServerStats}()
    check(ccall((:rvf_server_stats_get, LIB), Cint, (Ptr{Cvoid}, Ref{RvfServerStats}), sv, st))
    st[]
end

end # module
