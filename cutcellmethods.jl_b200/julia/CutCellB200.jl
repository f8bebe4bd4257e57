# CutCellB200.jl -- the Julia side of the drop-in backend: CutCellMethods.jl's cache API
# (allocate_cache / update_cache! / the uniform readers) over libcutcell_b200.so.
#
# A `B200Backend()` cache keeps the reference's own types and layout: `cache.cells` is a
# StructArray of CutCellData whose columns are CuArrays, `cache.phi` (nodal methods) or
# `normals`/`intercepts`/`is_valid` (PLIC) stay where the reference keeps them. The library writes
# those device arrays through the C ABI in include/cutcell_b200.h; it never frees them. What the
# library owns (its op-tape buffer, tiling table, work lists, reduction scratch) hangs off a
# `cc_handle` freed by a finalizer.
#
# Not exercised in this repository's CI: the build container has no Julia. The Python mirror
# (cutcellmethods.jl_b200/cache.py) drives the same entry points in the tests.
module CutCellB200

using CUDA
using StructArrays
using StaticArrays
using CutCellMethods
using CutCellMethods: CutCellData, MarchingCubesCutCellCache, MarchingSquaresCutCellCache,
                      PLICCutCellCache, MarchingCubesCutCell, MarchingSquaresCutCell, PLICCutCell
using CartesianMeshes: CartesianGrid
import MarchingCubes
import SDFLibrary

export B200Backend

const LIB = get(ENV, "CUTCELL_B200_LIB", joinpath(@__DIR__, "..", "libcutcell_b200.so"))

struct B200Backend end

# ---- C ABI structs (include/cutcell_b200.h) -------------------------------------------------
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

const CC_OK, CC_DIM_MISMATCH, CC_ANISOTROPIC = 0, 1, 2

function check(status)
    status == CC_OK && return nothing
    msg = unsafe_string(ccall((:cc_last_error, LIB), Cstring, ()))
    status == CC_DIM_MISMATCH && throw(DimensionMismatch(msg))
    status in (CC_ANISOTROPIC, 3, 4, 7, 8, 9, 10) && throw(ArgumentError(msg))
    error("libcutcell_b200: [$status] $msg")
end

ccgrid(g::CartesianGrid{D}) where {D} =
    CCGrid(Int32(D), 0, ntuple(a -> a <= D ? Float64(g.x0[a]) : 0.0, 3),
           ntuple(a -> a <= D ? Float64(g.d[a]) : 1.0, 3), ntuple(a -> a <= D ? Int64(g.n[a]) : 1, 3))

ptr(a) = reinterpret(Ptr{Cvoid}, pointer(a))
cccells(c) = CCCells(ptr(c.kind), ptr(c.ambiguous), ptr(c.volume_fraction), ptr(c.centroid),
                     ptr(c.face_fraction), ptr(c.face_centroid_local), ptr(c.interface_centroid))

mutable struct Handle
    h::Ptr{Cvoid}
    function Handle(method, dim, prec, n::NTuple{3,Int64})
        out = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:cc_handle_create, LIB), Cint, (Int32, Int32, Int32, Int32, Ptr{Int64}, Ptr{Ptr{Cvoid}}),
                    CUDA.device().handle, method, dim, prec, Ref(n), out))
        x = new(out[])
        finalizer(x -> ccall((:cc_handle_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), x)
        return x
    end
end

precision(::Type{Float32}) = Int32(0)
precision(::Type{Float64}) = Int32(1)

# ---- bodies: SDFLibrary geometry flattened to the op-tape -----------------------------------
# Primitive layouts are those of include/cutcell_b200.h. SDFLibrary's field names are read as
# the reference's own tests read them (`center`, `radius`); other geometry types need a method
# of `emit!` here.
function flatten(geo, D)
    ops = CCOp[]; params = Float64[]
    prim!(op, vals, comb) = (push!(ops, CCOp(op, comb, length(params), 0, 0)); append!(params, vals))
    emit!(g::SDFLibrary.EmptyGeo, comb=0) = prim!(6, [1.0], comb)
    emit!(g::Union{SDFLibrary.SDFSphere,SDFLibrary.SDFCircle}, comb=0) =
        prim!(1, [Float64.(Tuple(g.center))..., Float64(g.radius)], comb)
    emit!(g, comb=0) = throw(ArgumentError("no op-tape form for $(typeof(g))"))
    emit!(geo)
    return ops, params
end

function with_tape(f, geo, D)
    ops, params = flatten(geo, D)
    GC.@preserve ops params begin
        t = CCOpTape(pointer(ops), length(ops), length(params), pointer(params))
        f(Ref(t))
    end
end

# ---- MarchingCubes.jl's Lewiner tables in the library's dispatch format ---------------------
# One entry per lookup index: the case number, the signed face tests, one outcome per
# combination of test results (optionally an interior test) and the tiling it selects -- the
# per-cube dispatch of src/marching_cubes/marching_cubes.jl:538-651, tabulated.
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

# ---- the cache API --------------------------------------------------------------------------
function CutCellMethods.allocate_cache(grid::CartesianGrid{3,T}, ::MarchingCubesCutCell;
                                       backend::B200Backend) where {T}
    n = Tuple(grid.n)
    h = Handle(Int32(1), Int32(3), precision(T), Int64.(n))
    blob = lewiner_table_blob()
    check(ccall((:cc_handle_set_mc_table, LIB), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Csize_t), h.h, blob, length(blob)))
    cols = ntuple(i -> CuArray{fieldtype(CutCellData{3,T,6,2}, i)}(undef, n), fieldcount(CutCellData{3,T,6,2}))
    cells = StructArray{CutCellData{3,T,6,2}}(NamedTuple{fieldnames(CutCellData{3,T,6,2})}(cols))
    cache = MarchingCubesCutCellCache(CuArray{T}(undef, n .+ 1), cells)
    HANDLES[objectid(cache)] = h
    return CutCellMethods.update_cache!(cache, SDFLibrary.EmptyGeo(one(T)), grid)
end

const HANDLES = IdDict{Any,Handle}()

function CutCellMethods.update_cache!(cache::MarchingCubesCutCellCache{<:CuArray}, geo, grid::CartesianGrid{3})
    h = HANDLES[objectid(cache)]
    g = Ref(ccgrid(grid)); c = Ref(cccells(cache.cells))
    with_tape(geo, 3) do t
        check(ccall((:cc_mc_update, LIB), Cint, (Ptr{Cvoid}, Ref{CCGrid}, Ptr{CCOpTape}, Ptr{Cvoid}, Ref{CCCells}, Ptr{Cvoid}),
                    h.h, g, t, ptr(cache.phi), c, CUDA.stream().handle))
    end
    CUDA.synchronize()
    return cache
end

end # module
