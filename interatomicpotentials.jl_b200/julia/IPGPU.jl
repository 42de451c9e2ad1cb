# IPGPU.jl — drop-in GPU evaluation for InteratomicPotentials.jl through libipg.so.
#
# Wrapping a potential in `GPU(...)` routes potential_energy / force / energy_and_force /
# virial_stress / virial and the SNAP descriptor functions to the CUDA library (include/ipg.h).
# Everything else (types, parameters, fitting code) stays the reference's.  Julia is not
# installed where this library was built, so this file has not been executed; it follows the
# C ABI declared in include/ipg.h one to one.
module IPGPU

using InteratomicPotentials, AtomsBase, StaticArrays, Unitful, UnitfulAtomic, ChainRulesCore
import InteratomicPotentials: energy_and_force, potential_energy, force, virial_stress, virial,
    compute_local_descriptors, compute_force_descriptors, compute_all_descriptors

const libipg = get(ENV, "IPG_LIBRARY", joinpath(@__DIR__, "..", "ipg", "libipg.so"))

struct IPGError <: Exception
    status::Cint
    msg::String
end

const Ctx = Ptr{Cvoid}
const _ctx = Ref{Ctx}(C_NULL)

function context()
    if _ctx[] == C_NULL
        h = Ref{Ctx}(C_NULL)
        st = ccall((:ipg_create, libipg), Cint, (Cint, Ref{Ctx}), 0, h)
        st == 0 || throw(IPGError(st, "ipg_create"))
        _ctx[] = h[]
    end
    _ctx[]
end

check(st, ctx = _ctx[]) = st == 0 || throw(IPGError(st,
    unsafe_string(ccall((:ipg_last_error, libipg), Cstring, (Ctx,), ctx))))

# ---- system -> flat arrays -------------------------------------------------------------
box(s) = [periodicity(s)[i] ? bounding_box(s)[i][i] : Inf * unit(bounding_box(s)[i][i]) for i in 1:3]
flatpos(s, strip) = reduce(vcat, [collect(strip.(p)) for p in position(s)])

# ---- pair potentials (ipg_pair_term, include/ipg.h) ----------------------------------------
struct PairTerm
    kind::Int32
    reserved::Int32
    coeff::Float64
    rcut::Float64
    species_mask::UInt64
    params::NTuple{8,Float64}
end

kind(::LennardJones) = 1;  params(p::LennardJones) = (p.ϵ, p.σ)
kind(::BornMayer) = 2;     params(p::BornMayer) = (p.A, p.ρ, p.σ, p.C, p.D)
kind(::Coulomb) = 3;       params(p::Coulomb) = (p.q₁, p.q₂)
kind(::Morse) = 4;         params(p::Morse) = (p.D, p.α, p.σ)
kind(::ZBL) = 5;           params(p::ZBL) = (Float64(p.Z₁), Float64(p.Z₂), p.e)

function term(p::EmpiricalPotential, c, syms)
    sp = get_species(p)
    mask = ismissing(sp) ? typemax(UInt64) :
        reduce(|, (UInt64(1) << (findfirst(==(s), syms) - 1) for s in sp if s in syms); init = UInt64(0))
    ps = params(p)
    PairTerm(kind(p), 0, c, get_rcutoff(p), mask, ntuple(i -> i <= length(ps) ? Float64(ps[i]) : 0.0, 8))
end
terms(p::EmpiricalPotential, syms) = [term(p, 1.0, syms)]
terms(p::LinearCombinationPotential, syms) =
    reduce(vcat, [[PairTerm(t.kind, 0, c * t.coeff, t.rcut, t.species_mask, t.params)
                   for t in terms(q, syms)] for (q, c) in zip(p.potentials, p.coefficients)])

struct GPU{P}
    p::P
end

function _pair(s, p)
    syms = unique(atomic_symbol(s))
    sp = Int32[findfirst(==(x), syms) - 1 for x in atomic_symbol(s)]
    ts = terms(p, syms)
    x = flatpos(s, austrip)
    L = austrip.(box(s))
    E, F, W = Ref(0.0), zeros(3length(s)), zeros(6)
    ctx = context()
    GC.@preserve x sp L ts F W begin
        check(ccall((:ipg_pair_eval, libipg), Cint,
                    (Ctx, Int64, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}, Ptr{PairTerm}, Int32,
                     Ref{Float64}, Ptr{Float64}, Ptr{Float64}, UInt32),
                    ctx, length(s), x, sp, L, ts, length(ts), E, F, W, 0x7))
    end
    E[], reinterpret(SVector{3,Float64}, F), SVector{6}(W)
end

function energy_and_force(s::AbstractSystem, g::GPU{<:Union{EmpiricalPotential,LinearCombinationPotential}})
    e, f, _ = _pair(s, g.p)
    (; e = e * u"hartree", f = f * u"hartree/bohr")
end
potential_energy(s::AbstractSystem, g::GPU) = energy_and_force(s, g).e
force(s::AbstractSystem, g::GPU) = energy_and_force(s, g).f
virial_stress(s::AbstractSystem, g::GPU{<:Union{EmpiricalPotential,LinearCombinationPotential}}) =
    _pair(s, g.p)[3] * u"hartree"
virial(s::AbstractSystem, g::GPU) = sum(virial_stress(s, g)[1:3])

# ---- SNAP (ipg_snap_params) -------------------------------------------------------------
struct SnapParams
    twojmax::Int32
    nspecies::Int32
    rcutfac::Float64
    rmin0::Float64
    rfac0::Float64
    radii::NTuple{8,Float64}
    weight::NTuple{8,Float64}
    chem_flag::Int32
    bzero_flag::Int32
    bnorm_flag::Int32
    switch_flag::Int32
    wselfall_flag::Int32
    literal_sqrt_radius::Int32
    quadratic_flag::Int32   # quadratic SNAP (the LAMMPS_SNAP keyword); the reference SNAP has none
    literal_chem_z::Int32   # compute_z.jl's own Z index with chem_flag
end

pad8(v) = ntuple(i -> i <= length(v) ? Float64(v[i]) : 0.0, 8)

function handle(snap::SNAP)
    p = SnapParams(snap.twojmax, length(snap.species), snap.rcutfac, snap.rmin0, snap.rfac0,
                   pad8(snap.radii), pad8(snap.weight), snap.chem_flag, snap.bzero_flag,
                   snap.bnorm_flag, snap.switch_flag, snap.wselfall_flag, 0, 0, 0)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:ipg_snap_create, libipg), Cint, (Ctx, Ref{SnapParams}, Ref{Ptr{Cvoid}}), context(), p, h))
    h[]
end

function compute_all_descriptors(A::AbstractSystem, g::GPU{<:SNAP})
    snap = g.p
    n, K, nsp = length(A), length(snap), length(snap.species)
    h = handle(snap)
    x = flatpos(A, ustrip)
    L = ustrip.(box(A))
    sp = Int32[findfirst(==(atomic_symbol(A, i)), snap.species) - 1 for i in 1:n]
    B, dB, W = zeros(K, n), zeros(3, K * nsp, n), zeros(6, K * nsp)
    GC.@preserve x L sp B dB W begin
        check(ccall((:ipg_snap_descriptors, libipg), Cint,
                    (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                     Ptr{Float64}, UInt32), h, n, x, sp, L, B, dB, W, 0x7))
    end
    ccall((:ipg_snap_destroy, libipg), Cint, (Ptr{Cvoid},), h)
    [B[:, i] for i in 1:n], [dB[:, :, i] for i in 1:n], W
end
compute_local_descriptors(A::AbstractSystem, g::GPU{<:SNAP}) = compute_all_descriptors(A, g)[1]
compute_force_descriptors(A::AbstractSystem, g::GPU{<:SNAP}) = compute_all_descriptors(A, g)[2]

# LBasisPotential over SNAP: energy and forces through the adjoint path (mode 1).
function energy_and_force(A::AbstractSystem, g::GPU{<:LBasisPotential})
    lbp = g.p
    snap = lbp.basis
    n, nsp = length(A), length(snap.species)
    h = handle(snap)
    x = flatpos(A, ustrip)
    L = ustrip.(box(A))
    sp = Int32[findfirst(==(atomic_symbol(A, i)), snap.species) - 1 for i in 1:n]
    β = repeat(lbp.β, nsp)  # one block per centre species, all equal to the reference's β
    E, F, W = Ref(0.0), zeros(3n), zeros(6)
    GC.@preserve x L sp β F W begin
        check(ccall((:ipg_snap_energy_forces, libipg), Cint,
                    (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}, Ptr{Float64}, Float64, Int32,
                     Ref{Float64}, Ptr{Float64}, Ptr{Float64}), h, n, x, sp, L, β, lbp.β0[1], 1, E, F, W))
    end
    ccall((:ipg_snap_destroy, libipg), Cint, (Ptr{Cvoid},), h)
    (; e = E[], f = reinterpret(SVector{3,Float64}, F))
end

# ---- pullbacks (ipg_snap_vjp, ipg_snap_batch_loss_grad) ----------------------------------
# Cotangents are taken in the library's units (energy as returned, positions in the system's
# length unit).  gE: cotangent of E; gF: cotangent of F (flat 3n, or nothing).
function snap_vjp(A::AbstractSystem, lbp::LBasisPotential, gE::Float64, gF)
    snap = lbp.basis
    n, K, nsp = length(A), length(snap), length(snap.species)
    h = handle(snap)
    x = flatpos(A, ustrip)
    L = ustrip.(box(A))
    sp = Int32[findfirst(==(atomic_symbol(A, i)), snap.species) - 1 for i in 1:n]
    β = repeat(lbp.β, nsp)
    gβ, gβ0, gx = zeros(K * nsp), Ref(0.0), zeros(3n)
    g = gF === nothing ? C_NULL : convert(Vector{Float64}, gF)
    GC.@preserve x L sp β g gβ gx begin
        check(ccall((:ipg_snap_vjp, libipg), Cint,
                    (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}, Ptr{Float64}, Float64,
                     Ptr{Float64}, Ptr{Float64}, Ref{Float64}, Ptr{Float64}),
                    h, n, x, sp, L, β, gE, g, gβ, gβ0, gx))
    end
    ccall((:ipg_snap_destroy, libipg), Cint, (Ptr{Cvoid},), h)
    # the reference's beta is one K-vector shared by every species block
    sum(reshape(gβ, K, nsp); dims = 2)[:, 1], gβ0[], reinterpret(SVector{3,Float64}, gx)
end

function ChainRulesCore.rrule(::typeof(potential_energy), A::AbstractSystem, g::GPU{<:LBasisPotential})
    e = potential_energy(A, g)
    function pullback(ē)
        gβ, gβ0, gx = snap_vjp(A, g.p, Float64(ustrip(ē)), nothing)
        (NoTangent(), Tangent{typeof(A)}(; position = gx),
         Tangent{typeof(g)}(; p = Tangent{typeof(g.p)}(; β = gβ, β0 = [gβ0])))
    end
    e, pullback
end

function ChainRulesCore.rrule(::typeof(force), A::AbstractSystem, g::GPU{<:LBasisPotential})
    f = force(A, g)
    function pullback(f̄)
        gF = reduce(vcat, [collect(Float64.(ustrip.(v))) for v in unthunk(f̄)])
        gβ, _, gx = snap_vjp(A, g.p, 0.0, gF)
        (NoTangent(), Tangent{typeof(A)}(; position = gx), Tangent{typeof(g)}(; p = Tangent{typeof(g.p)}(; β = gβ)))
    end
    f, pullback
end

# Force-matching loss over a batch: L = sum |F - F_ref|^2 and dL/dβ in one call
# (flattened configurations, one persistent evaluation).
function force_matching_loss(systems::Vector{<:AbstractSystem}, lbp::LBasisPotential, Fref::Vector{Float64})
    snap = lbp.basis
    K, nsp = length(snap), length(snap.species)
    h = handle(snap)
    off = Int64[0; cumsum(length.(systems))]
    x = reduce(vcat, [flatpos(s, ustrip) for s in systems])
    sp = Int32[findfirst(==(atomic_symbol(s, i)), snap.species) - 1 for s in systems for i in 1:length(s)]
    L = reduce(vcat, [ustrip.(box(s)) for s in systems])
    β = repeat(lbp.β, nsp)
    loss, gβ = Ref(0.0), zeros(K * nsp)
    GC.@preserve off x sp L β Fref gβ begin
        check(ccall((:ipg_snap_batch_loss_grad, libipg), Cint,
                    (Ptr{Cvoid}, Int32, Ptr{Int64}, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}, Ptr{Float64}, Float64,
                     Ptr{Float64}, Ref{Float64}, Ptr{Float64}),
                    h, length(systems), off, x, sp, L, β, lbp.β0[1], Fref, loss, gβ))
    end
    ccall((:ipg_snap_destroy, libipg), Cint, (Ptr{Cvoid},), h)
    loss[], sum(reshape(gβ, K, nsp); dims = 2)[:, 1]
end

function ChainRulesCore.rrule(::typeof(force_matching_loss), systems, lbp::LBasisPotential, Fref)
    l, gβ = force_matching_loss(systems, lbp, Fref)
    pullback(l̄) = (NoTangent(), NoTangent(), Tangent{typeof(lbp)}(; β = l̄ .* gβ), NoTangent())
    l, pullback
end

end # module
