# The B200 backend against CutCellMethods.jl's own host backend: what a maintainer runs wherever
# Julia, CUDA.jl, CutCellMethods.jl (with its pinned SDFLibrary, CartesianMeshes, MarchingCubes)
# and libcutcell_b200.so are present:
#
#     CUTCELL_B200_LIB=/path/to/libcutcell_b200.so julia --project=<env> test/runtests.jl
#
# It mirrors the reference's own device check (test/test_cache.jl:289-334: kinds exact, volume
# fractions within 100 eps(Float32), faces within 1e-4, shared faces single-valued, surfaces of
# equal size) with `backend=B200Backend()` in place of `CUDABackend()`, and adds what only a Julia
# session can check: that MarchingCubes.jl's tables encoded by `lewiner_table_blob` drive the
# kernels to the reference's moments on every sign pattern, and that the op-tape samples bodies as
# SDFLibrary does.
using Test, LinearAlgebra, StaticArrays, Random
using CUDA, KernelAbstractions, Adapt
using CutCellMethods, CartesianMeshes, SDFLibrary, MeshLibrary
include(joinpath(@__DIR__, "..", "CutCellB200.jl"))
using .CutCellB200

const G2 = CartesianIsoGrid(mincorner=(-1.2, -1.2), maxcorner=(1.2, 1.2), sz=0.05)
const G3 = CartesianIsoGrid(mincorner=(-1.2, -1.2, -1.2), maxcorner=(1.2, 1.2, 1.2), sz=0.1)
const CIRCLE = SDFCircle(center=SVector(0.013, -0.021), radius=0.83)
const SPHERE = SDFSphere(SVector(0.01, 0.02, -0.03), 1.0)

# the number of interior faces whose two cells disagree
function shared_face_mismatches(ff::AbstractArray{<:SVector})
    D = ndims(ff); bad = 0
    for ci in CartesianIndices(ff), a in 1:D
        cj = ci + CartesianIndex(ntuple(b -> b == a ? 1 : 0, D))
        checkbounds(Bool, ff, cj) || continue
        bad += ff[ci][2a] === ff[cj][2a-1] ? 0 : 1
    end
    return bad
end

@testset "CutCellB200" begin
    @testset "the host backend is untouched by loading the module" begin
        host = update_cache!(allocate_cache(G3, MarchingCubesCutCell()), SPHERE, G3)
        @test host.phi isa Array && count(==(CutCellMethods.CELL_CUT), host.cells.kind) > 0
        @test KernelAbstractions.get_backend(host) isa KernelAbstractions.CPU
    end

    @testset "B200 agrees with the host (test/test_cache.jl:289-334)" begin
        for (method, g, geo) in ((MarchingSquaresCutCell(), G2, CIRCLE), (MarchingCubesCutCell(), G3, SPHERE),
                                 (PLICCutCell(), G2, CIRCLE), (PLICCutCell(), G3, SPHERE))
            g32 = CartesianMeshes.adapt_type(Float32, g)
            geo32 = SDFLibrary.adapt_type(Float32, geo)
            host = update_cache!(allocate_cache(g32, method), geo32, g32)
            dev = update_cache!(allocate_cache(g32, method; backend=B200Backend()), geo32, g32)
            @test KernelAbstractions.get_backend(dev) isa B200Backend
            @test Array(dev.cells.kind) == host.cells.kind
            @test maximum(abs.(Array(dev.cells.volume_fraction) .- host.cells.volume_fraction)) < 100 * eps(Float32)
            @test maximum(f -> maximum(abs, f), Array(dev.cells.face_fraction) .- host.cells.face_fraction) < 1e-4
            @test shared_face_mismatches(Array(dev.cells.face_fraction)) == 0
            if method isa Union{MarchingCubesCutCell,MarchingSquaresCutCell}
                @test length(generate_mesh(dev, g32; warn=false).elements) ==
                      length(generate_mesh(host, g32; warn=false).elements) > 0
            end
        end
    end

    @testset "Float64 phi is SDFLibrary's sdf_value at get_node, bit for bit" begin
        for (g, geo) in ((G3, SPHERE), (G2, CIRCLE))
            M = ndims(g) == 3 ? MarchingCubesCutCell() : MarchingSquaresCutCell()
            host = update_cache!(allocate_cache(g, M), geo, g)
            dev = update_cache!(allocate_cache(g, M; backend=B200Backend()), geo, g)
            @test Array(dev.phi) == host.phi
        end
    end

    @testset "MarchingCubes.jl's tables through lewiner_table_blob: every sign pattern" begin
        # the 256 sign patterns x 4 magnitudes of test/test_mc_moments.jl:219-244, each cube
        # updated on both backends from the same corner values: the tiling decides vf, centroid
        # and interface centroid of a non-planar cell, so agreement pins the encoding
        g = CartesianGrid(SVector(0.0, 0.0, 0.0), (1, 1, 1), SVector(1.0, 1.0, 1.0))
        host = allocate_cache(g, MarchingCubesCutCell())
        dev = allocate_cache(g, MarchingCubesCutCell(); backend=B200Backend())
        bits = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))
        rng = MersenneTwister(20260919)
        worst = 0.0; ncut = 0
        for mask in 0:255, _ in 1:4
            phi = ntuple(k -> ((mask >> (k - 1)) & 1 == 1 ? 1 : -1) * (0.05 + rand(rng)), 8)
            vals = zeros(2, 2, 2)
            for k in 1:8; vals[1 .+ bits[k]...] = phi[k]; end
            f(x) = vals[round(Int, x[1]) + 1, round(Int, x[2]) + 1, round(Int, x[3]) + 1]
            update_cache!(host, f, g)
            update_cache!(dev, NodalValues(CuArray(vals)), g)
            h = host.cells[1]
            @test Array(dev.cells.kind)[1] == h.kind
            @test Array(dev.cells.ambiguous)[1] == h.ambiguous
            h.kind == CutCellMethods.CELL_CUT || continue
            ncut += 1
            worst = max(worst, abs(Array(dev.cells.volume_fraction)[1] - h.volume_fraction),
                        maximum(abs, Array(dev.cells.centroid)[1] - h.centroid),
                        maximum(abs, Array(dev.cells.interface_centroid)[1] - h.interface_centroid))
        end
        @test ncut == 254 * 4
        @test worst < 1e-12
    end

    @testset "the benchmarked bodies: the CSG union and the 64-sphere cloud" begin
        rng = MersenneTwister(0)
        q = normalize(randn(rng, 4)); w, x, y, z = q
        R = @SMatrix [1-2(y^2+z^2) 2(x*y-w*z) 2(x*z+w*y); 2(x*y+w*z) 1-2(x^2+z^2) 2(y*z-w*x); 2(x*z-w*y) 2(y*z+w*x) 1-2(x^2+y^2)]
        body = CSGUnion(SDFSphere(SVector{3}(0.1 .* rand(rng, 3) .- 0.05), 0.45),
                        Box(SVector(0.0, 0.0, 0.0), SVector(0.3, 0.2, 0.6)), Torus(SVector(0.0, 0.0, 0.0), 0.5, 0.12, R))
        g = CartesianGrid(SVector(-1.0, -1.0, -1.0), (64, 64, 64), SVector(2 / 64, 2 / 64, 2 / 64))
        host = update_cache!(allocate_cache(g, MarchingCubesCutCell()), body, g)
        dev = update_cache!(allocate_cache(g, MarchingCubesCutCell(); backend=B200Backend()), body, g)
        @test Array(dev.phi) == host.phi
        @test Array(dev.cells.kind) == host.cells.kind
        @test maximum(abs.(Array(dev.cells.volume_fraction) .- host.cells.volume_fraction)) < 1e-12
        cloud = CSGUnion((SDFSphere(SVector{3}(0.1 .+ 0.8 .* rand(rng, 3)), 0.02 + 0.06 * rand(rng)) for _ in 1:64)...)
        gu = CartesianGrid(SVector(0.0, 0.0, 0.0), (48, 48, 48), SVector(1 / 48, 1 / 48, 1 / 48))
        vh = calc_volume(cloud, gu); vd = calc_volume(cloud, gu, B200Backend())
        @test abs(vd - vh) < 1e-12 * max(1.0, abs(vh))
        p = update_cache!(allocate_cache(gu, PLICCutCell(); backend=B200Backend()), cloud, gu)
        @test shared_face_mismatches(Array(p.cells.face_fraction)) == 0
        @test length(generate_mesh(p, gu).elements) > 0
    end

    @testset "a tree cache on the device" begin
        MS = MarchingSquaresCutCell()
        base = CartesianGrid(mincorner=(-1.5, -1.5), maxcorner=(1.5, 1.5), n=(8, 8))
        tree = AdaptiveMesh(base; max_level=2, initial_level=1)
        CartesianMeshes.refine_where!(c -> CartesianMeshes.get_elem_centroid(tree, c)[1] > 0, tree)
        host = update_cache!(allocate_cache(tree, MS), CIRCLE, tree)
        dev = update_cache!(allocate_cache(tree, MS; backend=B200Backend()), CIRCLE, tree)
        @test Array(dev.cells.kind) == host.cells.kind
        @test maximum(abs.(Array(dev.cells.volume_fraction) .- host.cells.volume_fraction)) < 1e-13
        @test length(generate_mesh(dev, tree).elements) == length(generate_mesh(host, tree).elements) > 0
    end

    @testset "errors are the reference's" begin
        dev = allocate_cache(G3, MarchingCubesCutCell(); backend=B200Backend())
        g2 = CartesianIsoGrid(mincorner=(-1.0, -1.0, -1.0), maxcorner=(1.0, 1.0, 1.0), sz=0.25)
        @test_throws DimensionMismatch update_cache!(dev, SPHERE, g2)
        @test_throws ArgumentError update_cache!(dev, x -> x[1], G3)  # no op-tape form for a callable
    end
end
