# QED2d.jl -- Julia shim over libqed2d (the C ABI in include/qed2d.h) that keeps
# the exported API of the QED2d package (src/QED2d.jl:27-54).  Device arrays stay
# CuArrays in the package's own layout; each call passes their device pointers.
#
# Deviation: functions the package launches as kernels with
#   CUDA.@cuda threads=kprm.threads blocks=kprm.blocks f(args...)
# are ordinary functions here, called as f(args...); KernelParm is accepted and
# ignored.  CG non-convergence raises Base.error as in src/QED2dSolver.jl:98-102.
#
# Julia is not installed where this library is built and tested, so the shim is
# never run there.  tests/test_julia_shim.py reads it as text instead: its export
# list against the reference's, every ccall's symbol, argument and return types
# against include/qed2d.h, and the C struct mirrors field by field.  The entry
# points themselves run in the GPU tests through the Python mirror (qed2d/).
module QED2d

import CUDA, DelimitedFiles, LinearAlgebra, Random

const lib = get(ENV, "QED2D_LIB", joinpath(@__DIR__, "..", "lib", "libqed2d.so"))

struct LattParm
    iL::Tuple{Int64,Int64}
    beta::Float64
end
struct KernelParm
    threads::Tuple{Int64,Int64}
    blocks::Tuple{Int64,Int64}
end
mutable struct RHMCParm
    r_b::Float64
    n::Int64
    eps::Float64
    A::Float64
    rho::Vector{Float64}
    mu::Vector{Float64}
    nu::Vector{Float64}
    delta::Float64
    reweighting_N::Int64
    reweighting_Taylor::Int64
end
abstract type Integrators end
struct Leapfrog <: Integrators end
struct OMF4 <: Integrators end
export LattParm, KernelParm, RHMCParm, Integrators, Leapfrog, OMF4

# C struct qed2d_rhmc_params
struct CRhmc
    r_b::Cdouble; n::Int32; eps::Cdouble; A::Cdouble
    rho::NTuple{32,Cdouble}; mu::NTuple{32,Cdouble}; nu::NTuple{32,Cdouble}
    delta::Cdouble; reweighting_N::Int32; reweighting_Taylor::Int32
end
pad32(v) = ntuple(i -> i <= length(v) ? Float64(v[i]) : 0.0, 32)
CRhmc(r::RHMCParm) = CRhmc(r.r_b, r.n, r.eps, r.A, pad32(r.rho), pad32(r.mu), pad32(r.nu), r.delta,
                          r.reweighting_N, r.reweighting_Taylor)
struct CHmcResult
    accepted::Int32; hini::Cdouble; hfin::Cdouble; dH::Cdouble; qtop::Cdouble; cg_iterations::Int64
end

const CTX = Dict{Tuple{Int,Int,Int},Ptr{Cvoid}}()
const SEED = Ref{UInt64}(1234)
const COUNTER = Ref{UInt32}(0)
seed!(s) = (SEED[] = UInt64(s); COUNTER[] = 0; nothing)
next_counter() = (c = COUNTER[]; COUNTER[] += UInt32(1); c)

function check(st, what)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:qed2d_last_error, lib), Cstring, ()))
    st == 1 && Base.error("CG not converged ($what): $msg")
    Base.error("$what: $msg (status $st)")
end

function ctx(prm::LattParm)
    key = (prm.iL[1], prm.iL[2], CUDA.deviceid(CUDA.device()))
    h = get!(CTX, key) do
        p = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:qed2d_ctx_create, lib), Cint, (Cint, Cint, Cdouble, Ptr{Ptr{Cvoid}}),
                    prm.iL[1], prm.iL[2], prm.beta, p), "ctx_create")
        p[]
    end
    ccall((:qed2d_ctx_set_beta, lib), Cint, (Ptr{Cvoid}, Cdouble), h, prm.beta)
    ccall((:qed2d_ctx_set_stream, lib), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), h, CUDA.stream().handle)
    return h
end
set_precision!(prm::LattParm, p::Integer) = check(ccall((:qed2d_ctx_set_precision, lib), Cint,
                                                        (Ptr{Cvoid}, Cint), ctx(prm), p), "set_precision")
# CUDA-graph replay of HMC!'s MD integration on this lattice's context (on by default)
set_graphs!(prm::LattParm, on::Bool) = check(ccall((:qed2d_ctx_set_graphs, lib), Cint,
                                                   (Ptr{Cvoid}, Cint), ctx(prm), on ? 1 : 0), "set_graphs")

const CF = CuArray{ComplexF64}
const RF = CuArray{Float64}
dptr(a) = reinterpret(CUDA.CuPtr{Cdouble}, pointer(a))   # device pointer of a CuArray

# ---- gauge kernels: src/QED2dAction.jl ----
plaquette!(plx::RF, U::CF, prm::LattParm) =
    check(ccall((:qed2d_plaquette_field, lib), Cint, (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}),
                ctx(prm), dptr(plx), dptr(U)), "plaquette!")
qtop!(plx::RF, U::CF, prm::LattParm) =
    check(ccall((:qed2d_qtop_field, lib), Cint, (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}),
                ctx(prm), dptr(plx), dptr(U)), "qtop!")
krnl_force!(frc1::RF, frc2::RF, U::CF, prm::LattParm) =
    check(ccall((:qed2d_krnl_force, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}),
                ctx(prm), dptr(frc1), dptr(frc2), dptr(U)), "krnl_force!")
updt_fld!(U::CF, mom::RF, eps) =
    check(ccall((:qed2d_updt_fld, lib), Cint, (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble),
                ctx(LattParm((size(U, 1), size(U, 2)), 0.0)), dptr(U), dptr(mom), eps), "updt_fld!")
export plaquette!, qtop!, updt_fld!, krnl_force!

# ---- Dirac operator: src/QED2dDirac.jl ----
for (jl, c) in ((:gamm5Dw, :qed2d_gamm5dw), (:Dw, :qed2d_dw), (:gamm5Dw_sqr, :qed2d_gamm5dw_sqr),
                (:gamm5Dw_sqr_sqr, :qed2d_gamm5dw_sqr_sqr))
    @eval $jl(so::CF, U::CF, si::CF, am0, prm::LattParm, kprm=nothing) =
        check(ccall(($(QuoteNode(c)), lib), Cint,
                    (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble),
                    ctx(prm), dptr(so), dptr(U), dptr(si), am0), $(string(jl)))
end
gamm5Dw_sqr_msq(so::CF, tmp, U::CF, si::CF, am0, prm::LattParm, kprm=nothing) = gamm5Dw_sqr(so, U, si, am0, prm)
gamm5Dw_sqr_musq(so::CF, tmp, U::CF, si::CF, am0, mu, prm::LattParm, kprm=nothing) =
    check(ccall((:qed2d_gamm5dw_sqr_musq, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble, Cdouble),
                ctx(prm), dptr(so), dptr(U), dptr(si), am0, mu), "gamm5Dw_sqr_musq")
gamm5Dw_sqr_sqr_musq(so::CF, tmp, U::CF, si::CF, am0, mu, prm::LattParm, kprm=nothing) =
    check(ccall((:qed2d_gamm5dw_sqr_sqr_musq, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble, Cdouble),
                ctx(prm), dptr(so), dptr(U), dptr(si), am0, mu), "gamm5Dw_sqr_sqr_musq")
gamm5(so::CF, si::CF, am0, prm::LattParm) =
    check(ccall((:qed2d_gamm5, lib), Cint, (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}),
                ctx(prm), dptr(so), dptr(si)), "gamm5")
tr_dQwdU(frc::RF, U::CF, X::CF, g5DwX::CF, prm::LattParm) =
    check(ccall((:qed2d_tr_dqwdu, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}),
                ctx(prm), dptr(frc), dptr(U), dptr(X), dptr(g5DwX)), "tr_dQwdU")
export gamm5Dw, gamm5Dw_sqr, gamm5Dw_sqr_msq, tr_dQwdU, gamm5Dw_sqr_musq, gamm5Dw_sqr_sqr_musq,
       gamm5Dw_sqr_sqr, gamm5, Dw

# ---- CG: src/QED2dSolver.jl (both methods) ----
function CG(so::CF, U::CF, si::CF, am0, maxiter, eps, A, prm::LattParm, kprm)
    it = Ref{Cint}(0)
    check(ccall((:qed2d_cg, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble, Cint,
                 Cdouble, Ptr{Cint}), ctx(prm), dptr(so), dptr(U), dptr(si), am0, maxiter, eps, it), "CG")
    return Int(it[])
end
function CG(so::CF, U::CF, si::CF, am0, mu_mass, maxiter, eps, A, prm::LattParm, kprm; so_as_guess::Bool=false)
    it = Ref{Cint}(0)
    check(ccall((:qed2d_cg_shift, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble, Cdouble,
                 Cint, Cdouble, Cint, Ptr{Cint}),
                ctx(prm), dptr(so), dptr(U), dptr(si), am0, mu_mass, maxiter, eps, so_as_guess, it), "CG")
    return Int(it[])
end
export CG

# ---- observables: src/QED2dHMC.jl:198-237 ----
for (jl, c) in ((:Action, :qed2d_action), (:Plaquette, :qed2d_plaquette))
    @eval function $jl(U::CF, prm::LattParm, kprm=nothing)
        v = Ref{Cdouble}(0)
        check(ccall(($(QuoteNode(c)), lib), Cint, (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, Ptr{Cdouble}),
                    ctx(prm), dptr(U), v), $(string(jl)))
        return v[]
    end
end
function Qtop(U::CF, prm::LattParm, kprm=nothing)
    v = Ref{Cdouble}(0)
    check(ccall((:qed2d_qtop, lib), Cint, (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, Ptr{Cdouble}, Ptr{Int64}),
                ctx(prm), dptr(U), v, C_NULL), "Qtop")
    return v[]
end
function Hamiltonian(mom::RF, U::CF, prm::LattParm, kprm=nothing)
    v = Ref{Cdouble}(0)
    check(ccall((:qed2d_hamiltonian, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Ptr{Cdouble}), ctx(prm), dptr(mom), dptr(U), v),
          "Hamiltonian")
    return v[]
end

# ---- HMC: src/QED2dHMC.jl:19-195 ----
function push_result!(acc, r)
    push!(acc, Int(r.accepted))
    tag = r.accepted == 1 ? "ACCEPT" : "REJECT"
    @info("    $tag: Energy [inital: $(r.hini); final: $(r.hfin); difference: $(r.dH)]; Pacc = $(count(acc .== 1) / length(acc))")
end
function HMC!(U::CF, eps, ns, acc, prm::LattParm, kprm::KernelParm; integrator::Integrators=OMF4(), qzero=false)
    r = Ref{CHmcResult}()
    check(ccall((:qed2d_hmc_gauge, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, Cdouble, Cint, Cint, Cint, UInt64, UInt32, Ptr{CHmcResult}),
                ctx(prm), dptr(U), eps, ns, integrator isa OMF4 ? 1 : 0, qzero, SEED[], next_counter(), r), "HMC!")
    push_result!(acc, r[])
end
function HMC!(U::CF, am0, eps, ns, acc, CGmaxiter, tol, prm::LattParm, kprm::KernelParm;
              integrator::Integrators=Leapfrog(), qzero=false)
    r = Ref{CHmcResult}()
    check(ccall((:qed2d_hmc_nf2, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, Cdouble, Cdouble, Cint, Cint, Cint, Cdouble, Cint, UInt64, UInt32,
                 Ptr{CHmcResult}),
                ctx(prm), dptr(U), am0, eps, ns, integrator isa OMF4 ? 1 : 0, CGmaxiter, tol, qzero, SEED[],
                next_counter(), r), "HMC!")
    push_result!(acc, r[])
end
function HMC!(U::CF, am0::Array, eps, ns, acc, CGmaxiter, tol, prm::LattParm, kprm::KernelParm,
              rprm::Array{RHMCParm}; integrator::Integrators=Leapfrog(), qzero=false, reversibility_test=false)
    r = Ref{CHmcResult}()
    cr = [CRhmc(x) for x in rprm]
    check(ccall((:qed2d_hmc_rhmc, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, Cint, Ptr{Cdouble}, Cdouble, Cint, Cint, Cdouble, Ptr{CRhmc}, Cint,
                 Cint, UInt64, UInt32, Ptr{CHmcResult}),
                ctx(prm), dptr(U), length(am0), Float64.(am0), eps, ns, CGmaxiter, tol, cr, qzero, reversibility_test,
                SEED[], next_counter(), r), "HMC!")
    reversibility_test || push_result!(acc, r[])
    return nothing
end

# ---- molecular dynamics: src/QED2dHMC.jl:239-557 ----
const CPtrD = CUDA.CuPtr{Cdouble}
OMF4!(mom::RF, U::CF, eps, ns, prm::LattParm, kprm::KernelParm) =
    check(ccall((:qed2d_omf4_gauge, lib), Cint, (Ptr{Cvoid}, CPtrD, CPtrD, Cdouble, Cint),
                ctx(prm), dptr(mom), dptr(U), eps, ns), "OMF4!")
function OMF4!(mom::RF, U::CF, X::CF, F::CF, g5DX::CF, am0, eps, ns, maxiter, tol, prm::LattParm, kprm::KernelParm)
    it = Ref{Int64}(0)
    check(ccall((:qed2d_omf4_nf2, lib), Cint,
                (Ptr{Cvoid}, CPtrD, CPtrD, CPtrD, CPtrD, CPtrD, Cdouble, Cdouble, Cint, Cint, Cdouble, Ptr{Int64}),
                ctx(prm), dptr(mom), dptr(U), dptr(X), dptr(F), dptr(g5DX), am0, eps, ns, maxiter, tol, it), "OMF4!")
    return nothing
end
function leapfrog!(mom::RF, U::CF, X::CF, F::CF, g5DX::CF, am0, eps, ns, CGmaxiter, tol, prm::LattParm,
                   kprm::KernelParm)
    it = Ref{Int64}(0)
    check(ccall((:qed2d_leapfrog_nf2, lib), Cint,
                (Ptr{Cvoid}, CPtrD, CPtrD, CPtrD, CPtrD, CPtrD, Cdouble, Cdouble, Cint, Cint, Cdouble, Ptr{Int64}),
                ctx(prm), dptr(mom), dptr(U), dptr(X), dptr(F), dptr(g5DX), am0, eps, ns, CGmaxiter, tol, it), "leapfrog!")
    return nothing
end
# ns is accepted and unused, as in the reference (:452)
function update_momenta!(mom::RF, U::CF, X::CF, F::CF, g5DX::CF, am0, eps, ns, maxiter, tol, prm::LattParm,
                         kprm::KernelParm)
    check(ccall((:qed2d_update_momenta_nf2, lib), Cint,
                (Ptr{Cvoid}, CPtrD, CPtrD, CPtrD, CPtrD, CPtrD, Cdouble, Cdouble, Cint, Cdouble, Ptr{Int64}),
                ctx(prm), dptr(mom), dptr(U), dptr(X), dptr(F), dptr(g5DX), am0, eps, maxiter, tol, C_NULL), "update_momenta!")
    return nothing
end
# RHMC (:485-557): F holds one pseudofermion field per flavour
function leapfrog!(mom::RF, U::CF, X::CF, F::Vector, g5DX::CF, am0::Array, eps, ns, CGmaxiter, tol,
                   prm::LattParm, kprm::KernelParm, rprm::Array{RHMCParm})
    it = Ref{Int64}(0)
    Fp = CPtrD[dptr(f) for f in F]
    cr = [CRhmc(x) for x in rprm]
    check(ccall((:qed2d_leapfrog_rhmc, lib), Cint,
                (Ptr{Cvoid}, CPtrD, CPtrD, CPtrD, Ptr{CPtrD}, CPtrD, Cint, Ptr{Cdouble}, Cdouble, Cint, Cint,
                 Cdouble, Ptr{CRhmc}, Ptr{Int64}),
                ctx(prm), dptr(mom), dptr(U), dptr(X), Fp, dptr(g5DX), length(am0), Float64.(am0), eps, ns, CGmaxiter, tol,
                cr, it), "leapfrog!")
    return nothing
end
function update_momenta!(mom::RF, U::CF, X::CF, F::Vector, g5DX::CF, am0::Array, eps, ns, maxiter, tol,
                         prm::LattParm, kprm::KernelParm, rprm::Array{RHMCParm})
    it = Ref{Int64}(0)
    Fp = CPtrD[dptr(f) for f in F]
    cr = [CRhmc(x) for x in rprm]
    check(ccall((:qed2d_update_momenta_rhmc, lib), Cint,
                (Ptr{Cvoid}, CPtrD, CPtrD, CPtrD, Ptr{CPtrD}, CPtrD, Cint, Ptr{Cdouble}, Cdouble, Cint, Cdouble,
                 Ptr{CRhmc}, Ptr{Int64}),
                ctx(prm), dptr(mom), dptr(U), dptr(X), Fp, dptr(g5DX), length(am0), Float64.(am0), eps, maxiter, tol, cr, it),
          "update_momenta!")
    return Int(it[])   # CG iterations, as the reference's RHMC method returns
end
# the reference exports this spelling (src/QED2d.jl:36) and defines leapfrog!
const leapgrog! = leapfrog!
export HMC!, Hamiltonian, Action, Plaquette, Qtop, OMF4!, leapgrog!, update_momenta!, leapfrog!

# ---- RHMC: src/QED2dRHMC.jl ----
# Zolotarev helpers (:2-89), written on the library's Elliptic.K and Jacobi sn/cn
# (the reference calls Elliptic.jl for these, :3-5)
function ellipK(m)
    K = Ref{Cdouble}(0)
    check(ccall((:qed2d_ellip_K, lib), Cint, (Cdouble, Ptr{Cdouble}), m, K), "Elliptic.K")
    return K[]
end
function sncn(u, m)
    s, c = Ref{Cdouble}(0), Ref{Cdouble}(0)
    check(ccall((:qed2d_ellip_sncn, lib), Cint, (Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}), u, m, s, c),
          "Jacobi.sn/cn")
    return s[], c[]
end
k(eps) = sqrt(1.0 - eps)
v(n, eps) = ellipK(k(eps)^2) / (2.0 * n + 1.0)
a_r(r, n, eps) = (sc = sncn(r * v(n, eps), k(eps)^2); sc[2]^2 / sc[1]^2)
c_r(r, n, eps) = sncn(r * v(n, eps), k(eps)^2)[1]^2
mu(j, n, eps, r_b) = r_b * a_r(2 * j, n, eps)^(1 / 2)
nu(j, n, eps, r_b) = r_b * a_r(2 * j - 1, n, eps)^(1 / 2)
function rho_mu(j, k, l, n, eps, r_b)   # Luscher eq. (3.5)
    (j < k || j > l) && throw("j is not between k and l")
    res = nu(j, n, eps, r_b)^2 - mu(j, n, eps, r_b)^2
    for m in k:l
        m != j && (res *= (nu(m, n, eps, r_b)^2 - mu(j, n, eps, r_b)^2) / (mu(m, n, eps, r_b)^2 - mu(j, n, eps, r_b)^2))
    end
    return res
end
function rho_nu(j, k, l, n, eps, r_b)   # Luscher eq. (3.9)
    (j < k || j > l) && throw("j is not between k and l")
    res = mu(j, n, eps, r_b) - nu(j, n, eps, r_b)
    for m in k:l
        m != j && (res *= (mu(m, n, eps, r_b) - nu(j, n, eps, r_b)) / (nu(m, n, eps, r_b) - nu(j, n, eps, r_b)))
    end
    return res
end
function P(k, l, n, eps, r_b, Y)        # Luscher eq. (3.4)
    dim = size(Y, 2)
    res = LinearAlgebra.I(dim)
    if k != 0 && l != 0
        for j in k:l
            res = res .+ rho_mu(j, k, l, n, eps, r_b) * (Y .+ mu(j, n, eps, r_b)^2 * LinearAlgebra.I(dim))^(-1)
        end
    end
    println(res)
    return res
end
function d(n, eps)
    res = k(eps)^(2 * n + 1)
    for i in 1:2:2*n+1
        res *= c_r(i, n, eps)^2
    end
    return res
end
delta(n, eps) = d(n, eps)^2 / (1 + sqrt(1 - d(n, eps)^2))^2
function A(n, eps)
    res = 2 / (1 + sqrt(1 - d(n, eps)^2))
    for i in 1:2:2*n-1
        res *= c_r(i, n, eps)
    end
    for i in 2:2:2*n
        res *= 1 / c_r(i, n, eps)
    end
    return res
end
# shadows Base.error inside this module as in the reference; check() calls Base.error
error(Y, Yapprox) = abs(1 .- sqrt(Y) * Yapprox[1])
export k, v, a_r, c_r, mu, nu, rho_mu, P, d, A, delta, error

# LuscherZ (:174-186): Z = ((g5Dw)^2 R^2 - 1) X_in; LuscherZp (:189-202): p times
LuscherZ(Z::CF, U::CF, X_in::CF, am0, CGmaxiter, CGtol, rprm::RHMCParm, prm::LattParm, kprm=nothing) =
    check(ccall((:qed2d_luscher_z, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble, Cint, Cdouble,
                 Ref{CRhmc}), ctx(prm), dptr(Z), dptr(U), dptr(X_in), am0, CGmaxiter, CGtol, CRhmc(rprm)), "LuscherZ")
function LuscherZp(Z::CF, p::Int64, U::CF, X_in::CF, am0, CGmaxiter, CGtol, rprm::RHMCParm, prm::LattParm,
                   kprm=nothing)
    tmp = copy(X_in)
    for i in 1:p
        LuscherZ(Z, U, tmp, am0, CGmaxiter, CGtol, rprm, prm, kprm)
        tmp .= Z
    end
    return nothing
end
function get_rhmc_params(n::Int64, r_a, r_b; reweighting_N::Int64=1, reweighting_Taylor::Int64=5)
    c = Ref{CRhmc}()
    check(ccall((:qed2d_get_rhmc_params, lib), Cint, (Cint, Cdouble, Cdouble, Ptr{CRhmc}), n, r_a, r_b, c),
          "get_rhmc_params")
    x = c[]
    RHMCParm(x.r_b, x.n, x.eps, x.A, collect(x.rho[1:n]), collect(x.mu[1:n]), collect(x.nu[1:n]), x.delta,
             reweighting_N, reweighting_Taylor)
end
get_rhmc_params(n::Array, r_a::Array, r_b::Array; kw...) = [get_rhmc_params(n[j], r_a[j], r_b[j]) for j in 1:length(n)]
function power_method(U::CF, am0, prm, kprm; iter::Int64=1000)
    lmin, lmax = Ref{Cdouble}(0), Ref{Cdouble}(0)
    check(ccall((:qed2d_power_method, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, Cdouble, Cint, UInt64, UInt32, Ptr{Cdouble}, Ptr{Cdouble}),
                ctx(prm), dptr(U), am0, iter, SEED[], next_counter(), lmin, lmax), "power_method")
    return lmin[], lmax[]
end
for (jl, c) in ((:MultiCG, :qed2d_multi_cg), (:R, :qed2d_rational))
    @eval function $jl(so::CF, U::CF, si::CF, am0, maxiter, eps, A, rprm::RHMCParm, prm::LattParm, kprm=nothing)
        it = Ref{Cint}(0)
        check(ccall(($(QuoteNode(c)), lib), Cint,
                    (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble, Cint, Cdouble,
                     Ref{CRhmc}, Ptr{Cint}), ctx(prm), dptr(so), dptr(U), dptr(si), am0, maxiter, eps, CRhmc(rprm), it),
              $(string(jl)))
        return nothing
    end
end
function generate_pseudofermion!(F::CF, U::CF, X::CF, am0, CGmaxiter, CGtol, prm, kprm, rprm::RHMCParm)
    it = Ref{Cint}(0)
    check(ccall((:qed2d_generate_pseudofermion, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cdouble, Cint, Cdouble,
                 Ref{CRhmc}, Ptr{Cint}), ctx(prm), dptr(F), dptr(U), dptr(X), am0, CGmaxiter, CGtol, CRhmc(rprm), it),
          "generate_pseudofermion!")
end
function reweighting_factor(U::CF, am0, CGmaxiter, CGtol, prm::LattParm, kprm::KernelParm, rprm::RHMCParm)
    W = Ref{Cdouble}(0)
    check(ccall((:qed2d_reweighting_factor, lib), Cint,
                (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, Cdouble, Cint, Cdouble, Ref{CRhmc}, UInt64, UInt32, Ptr{Cdouble}),
                ctx(prm), dptr(U), am0, CGmaxiter, CGtol, CRhmc(rprm), SEED[], next_counter(), W), "reweighting_factor")
    return W[]
end
reweighting_factor(U, am0::Array{Float64}, CGmaxiter, CGtol, prm, kprm, rprm::Array{RHMCParm}) =
    prod(reweighting_factor(U, am0[j], CGmaxiter, CGtol, prm, kprm, rprm[j]) for j in 1:length(am0))
export get_rhmc_params, power_method, reweighting_factor, R, MultiCG, generate_pseudofermion!

# ---- fields, utilities, checkpoints ----
function unfold_fld!(Uin::CF, prm::LattParm, kprm=nothing; reflect=false)
    Uout = CUDA.ones(ComplexF64, 2 * prm.iL[1], 2 * prm.iL[2], 2)
    check(ccall((:qed2d_unfold, lib), Cint, (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, CUDA.CuPtr{Cdouble}, Cint),
                ctx(prm), dptr(Uout), dptr(Uin), reflect), "unfold")
    return Uout
end
unfold_reflect!(Uin::CF, prm::LattParm, kprm=nothing) = unfold_fld!(Uin, prm, kprm; reflect=true)
plwv(so::CF, k::Tuple{Float64,Float64}, prm::LattParm) =
    check(ccall((:qed2d_plwv, lib), Cint, (Ptr{Cvoid}, CUDA.CuPtr{Cdouble}, Cdouble, Cdouble),
                ctx(prm), dptr(so), k[1], k[2]), "plwv")
# checkpoints: one "Re<TAB>Im" line per link in column-major order (i1 fastest,
# then i2, then the direction) -- the text format of src/QED2dLoadSave.jl:1-19
function save_gauge(U, file::String, prm::LattParm)
    open(file, "w") do io
        for z in vec(Array(U))
            println(io, real(z), '\t', imag(z))
        end
    end
end
function load_gauge(U, file::String, prm::LattParm)
    rows = DelimitedFiles.readdlm(file, '\t', Float64)
    copyto!(U, reshape(complex.(rows[:, 1], rows[:, 2]), prm.iL[1], prm.iL[2], 2))
end
export unfold_fld!, unfold_reflect!, plwv, save_gauge, load_gauge

end # module
