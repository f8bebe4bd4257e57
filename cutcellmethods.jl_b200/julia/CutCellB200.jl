# CutCellB200.jl -- the Julia side of the drop-in backend: CutCellMethods.jl's own cache API
# (allocate_cache / update_cache! / generate_mesh / the uniform readers) over libcutcell_b200.so.
#
#     using CutCellMethods, CutCellB200
#     cache = allocate_cache(grid, MarchingCubesCutCell(); backend=B200Backend())
#     update_cache!(cache, geo, grid)          # libcutcell_b200.so, on the current CUDA device
#
# How it plugs in without replacing anything of the reference. The reference's keyword method
# `allocate_cache(grid, method; backend)` (src/marching_cubes/cache.jl:29-36,
# src/marching_squares/cache.jl:41-47,100-106, src/plic/cache.jl:60-75) allocates through two
# functions of the backend, `KernelAbstractions.allocate(backend, T, dims)` and
# `CutCellMethods._allocate_cells(backend, S, dims)`. This module adds methods of both for its own
# backend type, `B200Backend`: the first returns a `B200Array` (a CuArray plus the library handle of
# the cache it belongs to), the second a StructArray of plain CuArrays. So the cache the reference
# builds is its own struct type, with CuArray columns a consumer reads as a CUDABackend cache's,
# and with `phi` (nodal methods) or `normals`/`intercepts`/`is_valid` (PLIC) a `B200Array`. The
# `update_cache!` / `generate_mesh` methods below take caches parameterised on `B200Array` only:
# strictly more specific than the reference's methods, so they run for B200 caches and for nothing
# else -- CPU() and CUDABackend() caches keep the reference's own methods.
#
# The library handle (op-tape buffer, tiling table, work lists) lives in the `B200Array` that decides
# the cache's dispatch and is freed by that array's finalizer: no global table of handles.
#
# Not run in this repository: the build image has no Julia. `julia/test/runtests.jl` is the check a
# maintainer runs wherever Julia, CUDA.jl and CutCellMethods.jl are installed; the Python mirror
# (cutcellmethods.jl_b200/cache.py) drives the same C entry points in this repository's tests.
module CutCellB200

using CUDA
using StructArrays
using StaticArrays
import Adapt
import KernelAbstractions
using CutCellMethods
using CutCellMethods: CutCellData, MarchingCubesCutCellCache, MarchingSquaresCutCellCache, PLICCutCellCache,
                      MarchingCubesCutCell, MarchingSquaresCutCell, PLICCutCell
using CartesianMeshes: CartesianGrid, AdaptiveMesh, nleaves, leaf, get_elem_size
import MeshLibrary
using MeshLibrary: Mesh, Point, Tri, Line
import MarchingCubes
import SDFLibrary

export B200Backend, B200Array, NodalValues, Box, Torus, Plane3, CSGUnion, lewiner_table_blob, flatten

const LIB = get(ENV, "CUTCELL_B200_LIB", joinpath(@__DIR__, "..", "libcutcell_b200.so"))

# ---- status codes and C structs (include/cutcell_b200.h) -----------------------------------
const CC_OK, CC_DIM_MISMATCH, CC_ANISOTROPIC, CC_BACKEND_MISMATCH, CC_BAD_TAPE, CC_DEVICE_TIMEOUT,
      CC_CUDA_ERR, CC_BAD_ARG, CC_BAD_TABLE, CC_NO_TABLE, CC_TOO_LARGE, CC_BAD_FILE = 0:11
const CC_F32, CC_F64 = Int32(0), Int32(1)
const CC_MARCHING_SQUARES, CC_MARCHING_CUBES, CC_PLIC = Int32(0), Int32(1), Int32(2)

struct CCGrid
    dim::Int32; pad::Int32
    x0::NTuple{3,Float64}; d::NTuple{3,Float64}; n::NTuple{3,Int64}
end
struct CCCells
    kind::Ptr{Cvoid}; ambiguous::Ptr{Cvoid}; volume_fraction::Ptr{Cvoid}; centroid::Ptr{Cvoid}
    face_fraction::Ptr{Cvoid}; face_centroid_local::Ptr{Cvoid}; interface_centroid::Ptr{Cvoid}
end
struct CCOp
    opcode::UInt8; combine::UInt8; poff::UInt16; kparam::UInt16; reserved::UInt16
end
struct CCOpTape
    ops::Ptr{CCOp}; n_ops::Int32; n_params::Int32; params::Ptr{Float64}
end
struct CCTree
    x0::NTuple{2,Float64}; base_d::NTuple{2,Float64}; nleaves::Int64
    level::Ptr{Int32}; coord::Ptr{Int32}
end

"""Rethrow a library status as the reference's exception: `DimensionMismatch` for a grid that is
not the cache's (src/cache.jl:107-121), `ArgumentError` for bad input (src/plic/surface.jl:41-45)."""
function check(status)
    status == CC_OK && return nothing
    msg = unsafe_string(ccall((:cc_last_error, LIB), Cstring, ()))
    status == CC_DIM_MISMATCH && throw(DimensionMismatch(msg))
    status in (CC_ANISOTROPIC, CC_BACKEND_MISMATCH, CC_BAD_TAPE, CC_BAD_ARG, CC_BAD_TABLE, CC_NO_TABLE,
               CC_TOO_LARGE, CC_BAD_FILE) && throw(ArgumentError(msg))
    error("libcutcell_b200: [$status] $msg")
end

ccgrid(g::CartesianGrid{D}) where {D} =
    CCGrid(Int32(D), Int32(0), ntuple(a -> a <= D ? Float64(g.x0[a]) : 0.0, 3),
           ntuple(a -> a <= D ? Float64(g.d[a]) : 1.0, 3), ntuple(a -> a <= D ? Int64(g.n[a]) : Int64(1), 3))

devptr(a::CuArray) = reinterpret(Ptr{Cvoid}, pointer(a))
stream_handle() = reinterpret(Ptr{Cvoid}, CUDA.stream().handle)
precision_code(::Type{Float32}) = CC_F32
precision_code(::Type{Float64}) = CC_F64

# ---- the library handle of one cache ------------------------------------------------------
mutable struct Handle
    h::Ptr{Cvoid}
    function Handle(method::Int32, dim::Integer, ::Type{T}, n::NTuple{3,Int64}) where {T}
        out = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:cc_handle_create, LIB), Cint, (Int32, Int32, Int32, Int32, Ptr{Int64}, Ptr{Ptr{Cvoid}}),
                    Int32(CUDA.deviceid(CUDA.device())), method, Int32(dim), precision_code(T), Ref(n), out))
        x = new(out[])
        finalizer(x) do y
            y.h == C_NULL || ccall((:cc_handle_destroy, LIB), Cint, (Ptr{Cvoid},), y.h)
            y.h = C_NULL
        end
        return x
    end
end

# ---- the backend and its array type --------------------------------------------------------
"""
    B200Backend()

The backend to pass as `allocate_cache(grid, method; backend=B200Backend())`: the cache's updates,
`generate_mesh` and `calc_volume(geo, grid, B200Backend())` run in libcutcell_b200.so on the current
CUDA device. Its columns are CuArrays.
"""
struct B200Backend <: KernelAbstractions.GPU end

"""
    B200Array{T,N}

A CuArray that marks the cache holding it as a B200 cache, and holds that cache's library handle
(created at the cache's first update, freed with the array). `phi` of a nodal cache and the plane
arrays of a PLIC cache are `B200Array`s; `parent(a)` is the CuArray.
"""
mutable struct B200Array{T,N} <: AbstractArray{T,N}
    data::CuArray{T,N}
    handle::Union{Nothing,Handle}
end
B200Array(data::CuArray{T,N}) where {T,N} = B200Array{T,N}(data, nothing)
Base.size(a::B200Array) = size(a.data)
Base.parent(a::B200Array) = a.data
Base.getindex(a::B200Array, i::Int...) = CUDA.@allowscalar a.data[i...]
Base.setindex!(a::B200Array, v, i::Int...) = (CUDA.@allowscalar a.data[i...] = v; a)
Base.fill!(a::B200Array, v) = (fill!(a.data, v); a)
Base.Array(a::B200Array) = Array(a.data)
Base.copyto!(dst::Array, src::B200Array) = copyto!(dst, src.data)
Base.copyto!(dst::B200Array, src::AbstractArray) = (copyto!(dst.data, src); dst)
Adapt.adapt_structure(to, a::B200Array) = Adapt.adapt(to, a.data)
KernelAbstractions.get_backend(::B200Array) = B200Backend()
KernelAbstractions.synchronize(::B200Backend) = CUDA.synchronize()
KernelAbstractions.allocate(::B200Backend, ::Type{T}, dims::Dims) where {T} = B200Array(CuArray{T}(undef, dims))

# The reference allocates a cache's StructArray through this internal function of the backend
# (src/cache.jl:101-105): here its columns are plain CuArrays.
CutCellMethods._allocate_cells(::B200Backend, ::Type{S}, dims::Dims) where {S} =
    StructArray{S}(NamedTuple{fieldnames(S)}(ntuple(i -> CuArray{fieldtype(S, i)}(undef, dims), fieldcount(S))))

cccells(c) = CCCells(devptr(c.kind), devptr(c.ambiguous), devptr(c.volume_fraction), devptr(c.centroid),
                     devptr(c.face_fraction), devptr(c.face_centroid_local), devptr(c.interface_centroid))

# The cache's handle, created on first use: method, dimension, precision, cells per axis.
function handle!(a::B200Array, method::Int32, dim::Integer, ::Type{T}, n) where {T}
    if a.handle === nothing
        # cells per axis; a marching-squares tree is (leaves, 0, 0)
        nn = length(n) == 1 ? (Int64(n[1]), Int64(0), Int64(0)) : ntuple(i -> i <= length(n) ? Int64(n[i]) : Int64(1), 3)
        h = Handle(method, dim, T, nn)
        if method == CC_MARCHING_CUBES
            blob = lewiner_table_blob()
            check(ccall((:cc_handle_set_mc_table, LIB), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Csize_t), h.h, blob, length(blob)))
        end
        a.handle = h
    end
    return a.handle
end

# Block on the cache's stream, as update_cache! does (src/marching_squares/cache.jl:62).
finish(::Handle) = CUDA.synchronize()

# ---- bodies: SDFLibrary geometry flattened to the op-tape ------------------------------------
# Opcodes and combine modes of include/cutcell_b200.h.
const OP_SPHERE, OP_BOX, OP_TORUS, OP_PLANE, OP_CONST = 1, 2, 3, 4, 6
const COMB_PUSH, COMB_MIN, COMB_MAX, COMB_SMIN, COMB_SUB, COMB_NEG = 0, 1, 2, 3, 4, 5

"""
    Box(center, halfwidths) / Torus(center, R, r, rotation) / Plane3(point, normal) / CSGUnion(geos...; smoothing=0)

Bodies with an exact op-tape form, for what the benchmarked configurations need beyond
SDFLibrary's sphere and circle: the axis-aligned box, the torus rotated by a matrix (body frame
`rotation * (x - center)`, tube about the frame's z axis), the plane `dot(normal, x - point)`, and
the union -- `smoothing > 0` the polynomial smooth minimum `min(a,b) - h^2 k/4`,
`h = max(k - |a-b|, 0)/k`. Each is an `SDFLibrary.AbstractSDFGeometry` whose `sdf_value` is the
op-tape's own expression, so the reference's CPU backend samples the same numbers.
"""
struct Box{D} <: SDFLibrary.AbstractSDFGeometry
    center::SVector{D,Float64}; halfwidths::SVector{D,Float64}
end
struct Torus <: SDFLibrary.AbstractSDFGeometry
    center::SVector{3,Float64}; R::Float64; r::Float64; rotation::SMatrix{3,3,Float64,9}
end
struct Plane3{D} <: SDFLibrary.AbstractSDFGeometry
    point::SVector{D,Float64}; normal::SVector{D,Float64}
end
struct CSGUnion{G<:Tuple} <: SDFLibrary.AbstractSDFGeometry
    geos::G; smoothing::Float64
end
CSGUnion(geos...; smoothing::Real=0.0) = CSGUnion(geos, Float64(smoothing))

function SDFLibrary.sdf_value(g::Box{D}, x) where {D}
    q = ntuple(a -> abs(x[a] - g.center[a]) - g.halfwidths[a], D)
    u = max(q[1], 0.0) * max(q[1], 0.0)
    for a in 2:D; u = u + max(q[a], 0.0) * max(q[a], 0.0); end
    m = q[1]
    for a in 2:D; m = q[a] > m ? q[a] : m; end
    return sqrt(u) + (m < 0 ? m : 0.0)
end
function SDFLibrary.sdf_value(g::Torus, x)
    R = g.rotation
    d = (x[1] - g.center[1], x[2] - g.center[2], x[3] - g.center[3])
    l1 = (R[1, 1] * d[1] + R[1, 2] * d[2]) + R[1, 3] * d[3]
    l2 = (R[2, 1] * d[1] + R[2, 2] * d[2]) + R[2, 3] * d[3]
    l3 = (R[3, 1] * d[1] + R[3, 2] * d[2]) + R[3, 3] * d[3]
    qx = sqrt(l1 * l1 + l2 * l2) - g.R
    return sqrt(qx * qx + l3 * l3) - g.r
end
function SDFLibrary.sdf_value(g::Plane3{D}, x) where {D}
    s = g.normal[1] * (x[1] - g.point[1])
    for a in 2:D; s = s + g.normal[a] * (x[a] - g.point[a]); end
    return s
end
function SDFLibrary.sdf_value(g::CSGUnion, x)
    top = SDFLibrary.sdf_value(g.geos[1], x)
    for i in 2:length(g.geos)
        v = SDFLibrary.sdf_value(g.geos[i], x)
        if g.smoothing > 0
            k = g.smoothing
            h = max(k - abs(top - v), 0.0) / k
            top = (v < top ? v : top) - ((h * h) * k) * 0.25
        else
            top = v < top ? v : top
        end
    end
    return top
end

"""
    flatten(geo, D) -> (ops::Vector{CCOp}, params::Vector{Float64})

The op-tape of `geo`. Exact for SDFLibrary's `EmptyGeo`, `SDFSphere` and `SDFCircle` (fields
`center`, `radius`, as the reference's tests read them) and this module's `Box`, `Torus`, `Plane3`
and `CSGUnion`. SDFLibrary's `SDFPlane` and `SDFUnion` are read from their keyword names (`point`,
`normal`; `smoothing` and the member geometries) when their fields carry those names; anything
else is an `ArgumentError` -- there is no fallback that samples a callable on the host.
"""
function flatten(geo, D::Integer)
    ops = CCOp[]; params = Float64[]
    function prim!(op, vals, comb)
        push!(ops, CCOp(UInt8(op), UInt8(comb), UInt16(length(params)), UInt16(0), UInt16(0)))
        append!(params, Float64.(vals))
    end
    function combine!(comb, k)
        if comb == COMB_SMIN
            push!(params, Float64(k))
            push!(ops, CCOp(UInt8(0), UInt8(comb), UInt16(0), UInt16(length(params) - 1), UInt16(0)))
        else
            push!(ops, CCOp(UInt8(0), UInt8(comb), UInt16(0), UInt16(0), UInt16(0)))
        end
    end
    function emit!(g)
        if g isa SDFLibrary.EmptyGeo
            v = fieldcount(typeof(g)) >= 1 && getfield(g, 1) isa Real ? Float64(getfield(g, 1)) : 1.0
            prim!(OP_CONST, [v], COMB_PUSH)
        elseif g isa Union{SDFLibrary.SDFSphere,SDFLibrary.SDFCircle}
            length(g.center) == D || throw(ArgumentError("a $(length(g.center))D body on a $(D)D grid"))
            prim!(OP_SPHERE, [Tuple(g.center)..., g.radius], COMB_PUSH)
        elseif g isa Box
            prim!(OP_BOX, [Tuple(g.center)..., Tuple(g.halfwidths)...], COMB_PUSH)
        elseif g isa Torus
            D == 3 || throw(ArgumentError("a torus needs a 3D grid"))
            R = g.rotation
            prim!(OP_TORUS, [Tuple(g.center)..., (R[i, j] for i in 1:3 for j in 1:3)..., g.R, g.r], COMB_PUSH)
        elseif g isa Plane3
            prim!(OP_PLANE, [Tuple(g.point)..., Tuple(g.normal)...], COMB_PUSH)
        elseif g isa CSGUnion
            emit!(g.geos[1])
            for m in g.geos[2:end]
                emit!(m)
                g.smoothing > 0 ? combine!(COMB_SMIN, g.smoothing) : combine!(COMB_MIN, 0.0)
            end
        elseif g isa SDFLibrary.SDFPlane && hasfield(typeof(g), :point) && hasfield(typeof(g), :normal)
            prim!(OP_PLANE, [Tuple(g.point)..., Tuple(g.normal)...], COMB_PUSH)
        elseif g isa SDFLibrary.SDFUnion && hasfield(typeof(g), :smoothing)
            members = Any[]
            for f in fieldnames(typeof(g))
                v = getfield(g, f)
                v isa SDFLibrary.AbstractSDFGeometry && push!(members, v)
                v isa Union{Tuple,AbstractVector} && append!(members, filter(m -> m isa SDFLibrary.AbstractSDFGeometry, collect(v)))
            end
            isempty(members) && throw(ArgumentError("cannot find the members of $(typeof(g)) ($(fieldnames(typeof(g))))"))
            emit!(CSGUnion(Tuple(members), Float64(g.smoothing)))
        else
            throw(ArgumentError("CutCellB200 has no op-tape form for $(typeof(g)); use its Box, Torus, Plane3 " *
                                "or CSGUnion, or SDFLibrary's sphere / circle"))
        end
        return nothing
    end
    emit!(geo)
    return ops, params
end

function with_tape(f, geo, D)
    ops, params = flatten(geo, D)
    GC.@preserve ops params begin
        t = CCOpTape(pointer(ops), Int32(length(ops)), Int32(length(params)),
                     isempty(params) ? Ptr{Float64}(C_NULL) : pointer(params))
        return f(Ref(t))
    end
end

"""
    NodalValues(vals::CuArray)

A nodal field given by its values (sized `grid.n .+ 1`, or those values flattened), for
`update_cache!(cache, NodalValues(vals), grid)` on a marching-cubes or marching-squares B200 cache:
the cell pass alone, `phi` copied from `vals` (the reference's tests reach the same with a callable
that looks the node up).
"""
struct NodalValues{A<:CuArray}
    vals::A
end

# ---- MarchingCubes.jl's Lewiner tables in the library's dispatch format ---------------------
# One entry per lookup index: the case number, the signed face tests, one outcome per
# combination of test results (optionally an interior test) and the tiling it selects -- the
# per-cube dispatch of src/marching_cubes/marching_cubes.jl:538-651, tabulated. The encoding is
# checked end to end by julia/test/runtests.jl against the reference's own host backend, which
# reads the same tables through MarchingCubes.jl directly.
function lewiner_table_blob()
    MC = MarchingCubes
    luts = NTuple{4,Any}[]; outs = NTuple{5,Int}[]; tiles = Vector{Vector{Int8}}(); index = Dict{Vector{Int8},Int}()
    tile(t, n) = (v = Int8[t[i] for i in 1:3n]; get!(() -> (push!(tiles, v); length(tiles) - 1), index, v))
    out!(tt, tf=tt; itype=0, edge=0, s=0) = push!(outs, (itype, edge, s, tt, tf))
    for lut in 1:256
        case, cfg = Int(MC.cases[lut][1]), Int(MC.cases[lut][2])
        base = length(outs); faces = Int[]
        if case == 1
            out!(tile((), 0))
        elseif case in (2, 3, 6, 9, 10, 12, 15)
            tbl, n = Dict(2 => (MC.tiling1, 1), 3 => (MC.tiling2, 2), 6 => (MC.tiling5, 3), 9 => (MC.tiling8, 2),
                          10 => (MC.tiling9, 4), 12 => (MC.tiling11, 4), 15 => (MC.tiling14, 4))[case]
            out!(tile(tbl[cfg], n))
        elseif case == 4
            faces = [MC.test3[cfg]]
            out!(tile(MC.tiling3_1[cfg], 2)); out!(tile(MC.tiling3_2[cfg], 4))
        elseif case == 5
            out!(tile(MC.tiling4_1[cfg], 2), tile(MC.tiling4_2[cfg], 6); itype=1, s=MC.test4[cfg])
        elseif case == 7
            faces = [MC.test6[cfg][1]]
            out!(tile(MC.tiling6_1_1[cfg], 3), tile(MC.tiling6_1_2[cfg], 9); itype=2, edge=MC.test6[cfg][3], s=MC.test6[cfg][2])
            out!(tile(MC.tiling6_2[cfg], 5))
        elseif case == 8
            faces = [MC.test7[cfg][1], MC.test7[cfg][2], MC.test7[cfg][3]]
            for o in 0:7
                sub = o + 1
                if sub == 1; out!(tile(MC.tiling7_1[cfg], 3))
                elseif sub in (2, 3); out!(tile(MC.tiling7_2[cfg][sub-1], 5))
                elseif sub == 4; out!(tile(MC.tiling7_3[cfg][1], 9))
                elseif sub == 5; out!(tile(MC.tiling7_2[cfg][3], 5))
                elseif sub in (6, 7); out!(tile(MC.tiling7_3[cfg][sub-4], 9))
                else out!(tile(MC.tiling7_4_2[cfg], 9), tile(MC.tiling7_4_1[cfg], 5); itype=2, edge=MC.test7[cfg][5], s=MC.test7[cfg][4])
                end
            end
        elseif case in (11, 13)
            T = case == 11 ? MC.test10 : MC.test12
            faces = [T[cfg][1], T[cfg][2]]
            a, b, c = case == 11 ? (MC.tiling10_1_1, MC.tiling10_1_2, MC.tiling10_1_1_) : (MC.tiling12_1_1, MC.tiling12_1_2, MC.tiling12_1_1_)
            t2, t2_ = case == 11 ? (MC.tiling10_2, MC.tiling10_2_) : (MC.tiling12_2, MC.tiling12_2_)
            kw = case == 11 ? (itype=1, s=T[cfg][3]) : (itype=2, edge=T[cfg][4], s=T[cfg][3])
            out!(tile(a[cfg], 4), tile(b[cfg], 8); kw...)       # neither face test holds
            out!(tile(t2[cfg], 8))                              # first only
            out!(tile(t2_[cfg], 8))                             # second only
            out!(tile(c[cfg], 4))                               # both
        else # case == 14
            faces = [MC.test13[cfg][i] for i in 1:6]
            for o in 0:63
                sc = Int(MC.subcfg13[o + 1])
                if sc == 0; out!(tile(MC.tiling13_1[cfg], 4))
                elseif sc <= 6; out!(tile(MC.tiling13_2[cfg][sc], 6))
                elseif sc <= 18; out!(tile(MC.tiling13_3[cfg][sc-6], 10))
                elseif sc <= 22; out!(tile(MC.tiling13_4[cfg][sc-18], 12))
                elseif sc <= 26
                    sub = sc - 22
                    out!(tile(MC.tiling13_5_1[cfg][sub], 6), tile(MC.tiling13_5_2[cfg][sub], 10);
                         itype=2, edge=MC.tiling13_5_1[cfg][sub][1] - 1, s=MC.test13[cfg][6])
                elseif sc <= 38; out!(tile(MC.tiling13_3_[cfg][sc-26], 10))
                elseif sc <= 44; out!(tile(MC.tiling13_2_[cfg][sc-38], 6))
                else out!(tile(MC.tiling13_1_[cfg], 4))
                end
            end
        end
        push!(luts, (case, length(faces), faces, base))
    end
    io = IOBuffer()
    codes = reduce(vcat, tiles; init=Int8[])
    for (c, nt, f, b) in luts
        write(io, UInt8(c), UInt8(nt)); for i in 1:6; write(io, Int8(i <= nt ? f[i] : 0)); end
        write(io, UInt16(b), UInt16(0))
    end
    for (it, e, s, tt, tf) in outs; write(io, UInt8(it), UInt8(e), Int8(sign(s)), UInt8(0), UInt16(tt), UInt16(tf)); end
    off = 0
    for t in tiles; write(io, UInt16(off), UInt8(length(t) ÷ 3), UInt8(0)); off += length(t); end
    write(io, codes)
    body = take!(io)
    total = 24 + length(body); pad = (16 - total % 16) % 16
    hdr = reinterpret(UInt8, UInt32[0x544D4343, 1, length(outs), length(tiles), length(codes), total + pad])
    return vcat(hdr, body, zeros(UInt8, pad))
end

# ---- update_cache! for B200 caches ---------------------------------------------------------
# Each is strictly more specific than the reference's method for the same cache type (the first
# argument is parameterised on B200Array), so it is chosen for B200 caches only.

function CutCellMethods.update_cache!(cache::MarchingCubesCutCellCache{<:B200Array{T,3}}, geo,
                                      grid::CartesianGrid{3}) where {T}
    CutCellMethods._check_cache_size(cache.cells, grid)
    h = handle!(cache.phi, CC_MARCHING_CUBES, 3, T, size(cache.cells))
    g = Ref(ccgrid(grid)); c = Ref(cccells(cache.cells))
    if geo isa NodalValues
        length(geo.vals) == length(cache.phi) || throw(DimensionMismatch(
            "`vals` has $(length(geo.vals)) values but the grid has $(length(cache.phi)) nodes"))
        copyto!(vec(cache.phi.data), vec(T.(geo.vals)))
        check(ccall((:cc_mc_cells_from_phi, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{Cvoid}, Ref{CCCells}, Ptr{Cvoid}),
                    h.h, g, devptr(cache.phi.data), c, stream_handle()))
    else
        with_tape(geo, 3) do t
            check(ccall((:cc_mc_update, LIB), Cint,
                        (Ptr{Cvoid}, Ref{CCGrid}, Ptr{CCOpTape}, Ptr{Cvoid}, Ref{CCCells}, Ptr{Cvoid}),
                        h.h, g, t, devptr(cache.phi.data), c, stream_handle()))
        end
    end
    finish(h)
    return cache
end

function CutCellMethods.update_cache!(cache::MarchingSquaresCutCellCache{<:B200Array{T,2}}, geo,
                                      grid::CartesianGrid{2}) where {T<:Real}
    CutCellMethods._check_cache_size(cache.cells, grid)
    h = handle!(cache.phi, CC_MARCHING_SQUARES, 2, T, size(cache.cells))
    g = Ref(ccgrid(grid)); c = Ref(cccells(cache.cells))
    if geo isa NodalValues
        length(geo.vals) == length(cache.phi) || throw(DimensionMismatch(
            "`vals` has $(length(geo.vals)) values but the grid has $(length(cache.phi)) nodes"))
        copyto!(vec(cache.phi.data), vec(T.(geo.vals)))
        check(ccall((:cc_ms_cells_from_phi, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{Cvoid}, Ref{CCCells}, Ptr{Cvoid}),
                    h.h, g, devptr(cache.phi.data), c, stream_handle()))
    else
        with_tape(geo, 2) do t
            check(ccall((:cc_ms_update, LIB), Cint,
                        (Ptr{Cvoid}, Ref{CCGrid}, Ptr{CCOpTape}, Ptr{Cvoid}, Ref{CCCells}, Ptr{Cvoid}),
                        h.h, g, t, devptr(cache.phi.data), c, stream_handle()))
        end
    end
    finish(h)
    return cache
end

# A tree's leaves as the C ABI takes them: per leaf its level and integer coordinates at that
# level, with the leaf size base.d / 2^level -- checked against get_elem_size bit for bit, since
# the leaf kernel forms its corners x0 + T(coord + bit) * h from them
# (src/marching_squares/marching_squares.jl:113-121).
function tree_arrays(mesh::AdaptiveMesh{2,T}) where {T}
    n = nleaves(mesh)
    base_d = (Float64(mesh.base.d[1]), Float64(mesh.base.d[2]))
    level = Vector{Int32}(undef, n); coord = Vector{Int32}(undef, 2n)
    for i in 1:n
        c = leaf(mesh, i)
        h = get_elem_size(mesh, c)
        L = round(Int, log2(base_d[1] / Float64(h[1])))
        (T(base_d[1] / 2.0^L) == h[1] && T(base_d[2] / 2.0^L) == h[2]) || throw(ArgumentError(
            "leaf $i: its size $(Tuple(h)) is not the base cell size over 2^level"))
        level[i] = L; coord[2i-1] = c.coord[1]; coord[2i] = c.coord[2]
    end
    x0 = (Float64(mesh.base.x0[1]), Float64(mesh.base.x0[2]))
    return x0, base_d, CuArray(level), CuArray(coord)
end

function CutCellMethods.update_cache!(cache::MarchingSquaresCutCellCache{<:B200Array{SVector{4,T},1}}, geo,
                                      mesh::AdaptiveMesh{2}) where {T}
    n = nleaves(mesh)
    (length(cache.phi) == n && length(cache.cells) == n) || throw(DimensionMismatch(
        "the cache holds $(length(cache.cells)) leaves, but the tree has $n"))
    h = handle!(cache.phi, CC_MARCHING_SQUARES, 2, T, (n,))
    x0, base_d, level, coord = tree_arrays(mesh)
    c = Ref(cccells(cache.cells))
    with_tape(geo, 2) do t
        tr = Ref(CCTree(x0, base_d, Int64(n), reinterpret(Ptr{Int32}, pointer(level)), reinterpret(Ptr{Int32}, pointer(coord))))
        check(ccall((:cc_ms_tree_update, LIB), Cint,
                    (Ptr{Cvoid}, Ref{CCTree}, Ptr{CCOpTape}, Ptr{Cvoid}, Ref{CCCells}, Ptr{Cvoid}),
                    h.h, tr, t, devptr(cache.phi.data), c, stream_handle()))
    end
    finish(h)
    return cache
end

function CutCellMethods.update_cache!(cache::PLICCutCellCache{<:Any,<:Any,<:B200Array{T,D}},
                                      geo::SDFLibrary.AbstractSDFGeometry, grid::CartesianGrid{D}) where {T,D}
    CutCellMethods._check_cache_size(cache.cells, grid)
    CutCellMethods._require_isotropic(grid)
    h = handle!(cache.intercepts, CC_PLIC, D, T, size(cache.cells))
    g = Ref(ccgrid(grid)); c = Ref(cccells(cache.cells))
    with_tape(geo, D) do t
        check(ccall((:cc_plic_update, LIB), Cint,
                    (Ptr{Cvoid}, Ref{CCGrid}, Ptr{CCOpTape}, Ref{CCCells}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}),
                    h.h, g, t, c, devptr(parent(cache.normals)), devptr(cache.intercepts.data),
                    devptr(parent(cache.is_valid)), stream_handle()))
    end
    finish(h)
    return cache
end

# ---- generate_mesh for B200 caches: the surfaces built on the device --------------------------
# The same MeshLibrary types the reference returns (src/marching_cubes/surface.jl:82-112,
# src/marching_squares/surface.jl:59-108, src/plic/surface.jl:28-37), 1-based and dense. The
# geometry is the reference construction's; the numbering is the device's deterministic one (edge
# vertices by lower node then axis, triangles by cell), not MarchingCubes.march's.

function MeshLibrary.generate_mesh(cache::MarchingCubesCutCellCache{<:B200Array{T,3}}, grid::CartesianGrid{3};
                                   warn::Bool=true) where {T}
    h = handle!(cache.phi, CC_MARCHING_CUBES, 3, T, size(cache.cells))
    g = Ref(ccgrid(grid)); nv = Ref{Int64}(0); nt = Ref{Int64}(0)
    check(ccall((:cc_mc_mesh, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Int32}, Int64,
                                           Ptr{Int64}, Ref{Int64}, Ref{Int64}, Ptr{Cvoid}),
                h.h, g, devptr(cache.phi.data), C_NULL, 0, C_NULL, 0, C_NULL, nv, nt, stream_handle()))
    V = CuArray{T}(undef, 3, nv[]); F = CuArray{Int32}(undef, 3, nt[])
    check(ccall((:cc_mc_mesh, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Int32}, Int64,
                                           Ptr{Int64}, Ref{Int64}, Ref{Int64}, Ptr{Cvoid}),
                h.h, g, devptr(cache.phi.data), devptr(V), nv[], reinterpret(Ptr{Int32}, pointer(F)), nt[], C_NULL,
                nv, nt, stream_handle()))
    finish(h)
    warn && nt[] == 0 && @warn "no `sdf == 0` surface was found anywhere in `grid` -- returning an empty mesh."
    v = Array(V); f = Array(F)
    nodes = [Point(SVector{3,T}(v[1, i], v[2, i], v[3, i])) for i in 1:size(v, 2)]
    elements = [Tri(Int64(f[1, i]) + 1, Int64(f[2, i]) + 1, Int64(f[3, i]) + 1) for i in 1:size(f, 2)]
    return Mesh(nodes, elements)
end

function fetch_contour(h::Handle, ::Type{T}, nv, ns) where {T}
    V = CuArray{T}(undef, 2, nv); S = CuArray{Int32}(undef, 2, ns)
    check(ccall((:cc_ms_mesh_fetch, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Int32}, Ptr{Int64}, Ptr{Cvoid}),
                h.h, devptr(V), reinterpret(Ptr{Int32}, pointer(S)), C_NULL, stream_handle()))
    finish(h)
    v = Array(V); s = Array(S)
    nodes = [Point(SVector{2,T}(v[1, i], v[2, i])) for i in 1:size(v, 2)]
    elements = [Line(Int64(s[1, i]) + 1, Int64(s[2, i]) + 1) for i in 1:size(s, 2)]
    return Mesh(nodes, elements)
end

function MeshLibrary.generate_mesh(cache::MarchingSquaresCutCellCache{<:B200Array{T,2}}, grid::CartesianGrid{2};
                                   warn::Bool=true) where {T<:Real}
    h = handle!(cache.phi, CC_MARCHING_SQUARES, 2, T, size(cache.cells))
    nv = Ref{Int64}(0); ns = Ref{Int64}(0)
    check(ccall((:cc_ms_mesh_grid, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{Cvoid}, Ref{Int64}, Ref{Int64}, Ptr{Cvoid}),
                h.h, Ref(ccgrid(grid)), devptr(cache.phi.data), nv, ns, stream_handle()))
    warn && ns[] == 0 && @warn "no `sdf == 0` contour was found anywhere in `grid` -- returning an empty mesh."
    return fetch_contour(h, T, nv[], ns[])
end

function MeshLibrary.generate_mesh(cache::MarchingSquaresCutCellCache{<:B200Array{SVector{4,T},1}},
                                   mesh::AdaptiveMesh{2}; warn::Bool=true) where {T}
    h = handle!(cache.phi, CC_MARCHING_SQUARES, 2, T, (length(cache.cells),))
    x0, base_d, level, coord = tree_arrays(mesh)
    nv = Ref{Int64}(0); ns = Ref{Int64}(0)
    tr = Ref(CCTree(x0, base_d, Int64(nleaves(mesh)), reinterpret(Ptr{Int32}, pointer(level)),
                    reinterpret(Ptr{Int32}, pointer(coord))))
    check(ccall((:cc_ms_mesh_tree, LIB), Cint, (Ptr{Cvoid}, Ref{CCTree}, Ptr{Cvoid}, Ref{Int64}, Ref{Int64}, Ptr{Cvoid}),
                h.h, tr, devptr(cache.phi.data), nv, ns, stream_handle()))
    warn && ns[] == 0 && @warn "no `sdf == 0` contour was found anywhere in the tree -- returning an empty mesh."
    return fetch_contour(h, T, nv[], ns[])
end

function MeshLibrary.generate_mesh(cache::PLICCutCellCache{<:Any,<:Any,<:B200Array{T,D}}, grid::CartesianGrid{D};
                                   min_tri_area_fraction::Real=1e-4) where {T,D}
    CutCellMethods._check_cache_size(cache.cells, grid)
    h = handle!(cache.intercepts, CC_PLIC, D, T, size(cache.cells))
    g = Ref(ccgrid(grid)); nn = Ref{Int64}(0); ne = Ref{Int64}(0)
    args = (h.h, g, devptr(parent(cache.normals)), devptr(cache.intercepts.data), devptr(parent(cache.is_valid)),
            Float64(min_tri_area_fraction))
    check(ccall((:cc_plic_mesh, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble,
                                             Ptr{Cvoid}, Int64, Ptr{Int32}, Int64, Ptr{Int64}, Ref{Int64}, Ref{Int64},
                                             Ptr{Cvoid}),
                args..., C_NULL, 0, C_NULL, 0, C_NULL, nn, ne, stream_handle()))
    V = CuArray{T}(undef, D, nn[]); E = CuArray{Int32}(undef, D, ne[])
    check(ccall((:cc_plic_mesh, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble,
                                             Ptr{Cvoid}, Int64, Ptr{Int32}, Int64, Ptr{Int64}, Ref{Int64}, Ref{Int64},
                                             Ptr{Cvoid}),
                args..., devptr(V), nn[], reinterpret(Ptr{Int32}, pointer(E)), ne[], C_NULL, nn, ne, stream_handle()))
    finish(h)
    ne[] == 0 && @warn "no cut cell was found anywhere in `grid` -- returning an empty mesh."
    v = Array(V); e = Array(E)
    nodes = [Point(SVector{D,T}(ntuple(a -> v[a, i], D))) for i in 1:size(v, 2)]
    elements = D == 3 ? [Tri(Int64(e[1, i]) + 1, Int64(e[2, i]) + 1, Int64(e[3, i]) + 1) for i in 1:size(e, 2)] :
                        [Line(Int64(e[1, i]) + 1, Int64(e[2, i]) + 1) for i in 1:size(e, 2)]
    return Mesh(nodes, elements)
end

# ---- calc_volume on the device -----------------------------------------------------------
"""
    calc_volume(geo, grid, B200Backend()) -> T

`calc_volume(geo, grid)` (src/volume.jl:29-40) on the device: every cell's PLIC solid fraction,
summed in compensated Float64 and times `prod(grid.d)`, returned in the grid's element type.
"""
function CutCellMethods.calc_volume(geo::SDFLibrary.AbstractSDFGeometry, grid::CartesianGrid{D,T},
                                    ::B200Backend) where {D,T}
    CutCellMethods._require_isotropic(grid)
    h = Handle(CC_PLIC, D, T, ntuple(i -> i <= D ? Int64(grid.n[i]) : Int64(1), 3))
    out = Ref{Float64}(0.0)
    with_tape(geo, D) do t
        check(ccall((:cc_calc_volume, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{CCOpTape}, Ref{Float64}, Ptr{Cvoid}),
                    h.h, Ref(ccgrid(grid)), t, out, stream_handle()))
    end
    finalize(h)
    return T(out[])
end

end # module
