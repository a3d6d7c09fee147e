"""
    IPEPSB200

Julia binding of libipeps_b200 (include/ipeps_b200.h) for iPEPS.jl.

It mirrors the reference's hot-path API (src/ctm/ctmrg.jl, src/ctm/ctm_tensor.jl,
src/graph/evaluation.jl) so that iPEPS.jl can switch its bodies to the B200
engine when `cfg["backend"] == "b200"`:

    ts = CTMTensorsB200(A, cfg)             # CTMTensors(A, cfg): init_ctm1 on the device
    ts, conv = run_ctm(ts; conv_fun=H)      # run_ctm with the energy criterion
    E, Na = get_gs_energy(ts, H)
    E = ctm_energy(A, H, ts)                # differentiable: rrule -> ipeps_energy_grad

Arrays are column-major already, so they are passed as they are.  This file
is not exercised in this repository's tests (no Julia toolchain here); the
same C ABI is exercised through ctypes by the Python binding.
"""
module IPEPSB200

using ChainRulesCore

const lib = get(ENV, "IPEPS_B200_LIB", joinpath(@__DIR__, "..", "libipeps_b200.so"))

const IPEPS_CONV_ENERGY = Cint(0)
const IPEPS_CONV_SPECTRUM = Cint(1)

mutable struct Engine
    h::Ptr{Cvoid}
end

function check(ctx::Ptr{Cvoid}, st::Cint)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:ipeps_last_error, lib), Cstring, (Ptr{Cvoid},), ctx))
    error("libipeps_b200 status $st: $msg")
end

function Engine(device::Integer=0; precision::Symbol=:fp64)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    st = ccall((:ipeps_ctx_create, lib), Cint, (Cint, Ref{Ptr{Cvoid}}), device, r)
    st == 0 || error("ipeps_ctx_create failed ($st)")
    e = Engine(r[])
    check(e.h, ccall((:ipeps_ctx_set_precision, lib), Cint, (Ptr{Cvoid}, Cint), e.h, precision == :mixed ? 1 : 0))
    finalizer(x -> ccall((:ipeps_ctx_destroy, lib), Cint, (Ptr{Cvoid},), x.h), e)
    return e
end

const ENGINE = Ref{Union{Nothing,Engine}}(nothing)
engine() = (ENGINE[] === nothing && (ENGINE[] = Engine()); ENGINE[])

"""Device-side counterpart of `CTMTensors` (ctm_tensor.jl:3-18)."""
mutable struct CTMTensorsB200
    eng::Engine
    h::Ptr{Cvoid}
    A::Array{Float64,5}
    Params::Dict{String,Any}
end

function push_params!(ts::CTMTensorsB200)
    p = ts.Params
    check(ts.eng.h, ccall((:ipeps_env_set_params, lib), Cint, (Ptr{Cvoid}, Cint, Cint, Cint, Cint, Float64),
                          ts.h, get(p, "chi", 30), get(p, "min_iter", 4), get(p, "max_iter", 20),
                          get(p, "ad_max_iter", 4), get(p, "rg_tol", 1e-6)))
    # left/right and top/bottom moves on two streams (key absent: on)
    check(ts.eng.h, ccall((:ipeps_env_set_parallel, lib), Cint, (Ptr{Cvoid}, Cint),
                          ts.h, get(p, "parallel_moves", true) ? 1 : 0))
end

"""`CTMTensors(A, cfg)` (ctm_tensor.jl:63-69): Ad = conj(A), init_ctm1 on the device."""
function CTMTensorsB200(A::AbstractArray{Float64,5}, cfg::Dict; eng::Engine=engine())
    D, d = size(A, 1), size(A, 5)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(eng.h, ccall((:ipeps_env_create, lib), Cint, (Ptr{Cvoid}, Cint, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
                       eng.h, D, d, get(cfg, "chi", 30), 0, r))
    ts = CTMTensorsB200(eng, r[], Array{Float64,5}(A), copy(cfg))
    finalizer(x -> ccall((:ipeps_env_destroy, lib), Cint, (Ptr{Cvoid},), x.h), ts)
    push_params!(ts)
    GC.@preserve ts begin
        check(eng.h, ccall((:ipeps_env_set_A, lib), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}), ts.h, ts.A, C_NULL))
    end
    check(eng.h, ccall((:ipeps_env_init, lib), Cint, (Ptr{Cvoid},), ts.h))
    return ts
end

hmat(h) = Matrix{ComplexF64}(h)

"""`run_ctm(ts; conv_fun)` (ctmrg.jl:1-55).  Pass the Hamiltonian pair `H` as
`conv_fun` for the energy criterion (get_gs_energy), or `nothing` for the
spectrum criterion.  Returns (ts, last diff)."""
function run_ctm(ts::CTMTensorsB200; conv_fun=nothing)
    push_params!(ts)
    iters, diff, conv = Ref{Cint}(0), Ref{Float64}(0), Ref{Cint}(0)
    if conv_fun === nothing
        check(ts.eng.h, ccall((:ipeps_ctm_run, lib), Cint,
                              (Ptr{Cvoid}, Cint, Ptr{ComplexF64}, Ptr{ComplexF64}, Cint, Ref{Cint}, Ref{Float64}, Ref{Cint}),
                              ts.h, IPEPS_CONV_SPECTRUM, C_NULL, C_NULL, 0, iters, diff, conv))
    else
        Hh, Hv = hmat(conv_fun[1]), hmat(conv_fun[2])
        GC.@preserve Hh Hv begin
            check(ts.eng.h, ccall((:ipeps_ctm_run, lib), Cint,
                                  (Ptr{Cvoid}, Cint, Ptr{ComplexF64}, Ptr{ComplexF64}, Cint, Ref{Cint}, Ref{Float64}, Ref{Cint}),
                                  ts.h, IPEPS_CONV_ENERGY, Hh, Hv, size(Hh, 1), iters, diff, conv))
        end
    end
    conv[] == 0 && println("--------- Not Converged ----------")
    return ts, diff[]
end

"""`get_gs_energy(ts, H)` (evaluation.jl:15-29): (E, Na)."""
function get_gs_energy(ts::CTMTensorsB200, H)
    Hh, Hv = hmat(H[1]), hmat(H[2])
    E, Na = zeros(2), zeros(2)
    GC.@preserve Hh Hv E Na begin
        check(ts.eng.h, ccall((:ipeps_energy, lib), Cint,
                              (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{ComplexF64}, Cint, Ptr{Float64}, Ptr{Float64}),
                              ts.h, Hh, Hv, size(Hh, 1), E, Na))
    end
    return complex(E[1], E[2]), complex(Na[1], Na[2])
end

"""The pullback of `run_gs` (optim_gs.jl:133-143) from the environment held by ts."""
function energy_grad!(ts::CTMTensorsB200, H)
    Hh, Hv = hmat(H[1]), hmat(H[2])
    E = zeros(1)
    g = similar(ts.A)
    GC.@preserve Hh Hv E g begin
        check(ts.eng.h, ccall((:ipeps_energy_grad, lib), Cint,
                              (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{ComplexF64}, Cint, Cint, Ptr{Float64}, Ptr{Float64}),
                              ts.h, Hh, Hv, size(Hh, 1), get(ts.Params, "ad_max_iter", 4), E, g))
    end
    return E[1], g
end

"""
    ctm_energy(A, H, cfg)

`run_gs` of optim_gs.jl:133-143 as one differentiable function: converge from
init_ctm1, then ad_max_iter iterations + get_gs_energy.  Its rrule returns the
hand-written adjoint, so `Zygote.pullback(x -> ctm_energy(x, H, cfg), x)` in
fg! (optim_gs.jl:72) picks it up unchanged.
"""
function ctm_energy(A::AbstractArray{Float64,5}, H, cfg::Dict)
    ts = CTMTensorsB200(A, cfg)
    run_ctm(ts; conv_fun=H)
    E, _ = energy_grad!(ts, H)
    return E
end

function ChainRulesCore.rrule(::typeof(ctm_energy), A::AbstractArray{Float64,5}, H, cfg::Dict)
    ts = CTMTensorsB200(A, cfg)
    run_ctm(ts; conv_fun=H)
    E, g = energy_grad!(ts, H)
    ctm_energy_pullback(dE) = (NoTangent(), unthunk(dE) .* g, NoTangent(), NoTangent())
    return E, ctm_energy_pullback
end

end # module
