"""
    IPEPSB200

Julia binding of libipeps_b200 (include/ipeps_b200.h) for iPEPS.jl.

It mirrors the reference's hot-path API (src/ctm/ctmrg.jl, src/ctm/ctm_tensor.jl,
src/graph/evaluation.jl) so that iPEPS.jl can switch its bodies to the B200
engine when `cfg["backend"] == "b200"`:

    ts = CTMTensorsB200(A, cfg)             # CTMTensors(A, cfg): init_ctm1 on the device
    ts, conv = run_ctm(ts; conv_fun=H)      # run_ctm with the energy criterion
    E, Na = get_gs_energy(ts, H)
    E = ctm_energy(A, H, cfg)               # differentiable: rrule -> ipeps_energy_grad
    gH, gN = get_es_grad(ts1, H, Bi)        # get_es_grad (optim_es.jl:167-194) on a copy ts1

The excited-state unit of optim_es (optim_es.jl:127-153) per basis vector:

    ts1 = CTMTensorsB200(ts.A, ts.Params; init=false)
    for k in 1:4; set_CT!(ts1, k, get_CT(ts, k)...); end
    ts1.Params["px"], ts1.Params["py"] = px * pi, py * pi
    gH, gN = get_es_grad(ts1, H, basis[:, i])
    effH[:, i], effN[:, i] = basis' * gH / 2, basis' * gN

Arrays are column-major already, so they are passed as they are.  This file
is not exercised in this repository's tests (no Julia toolchain here); the
same C ABI is exercised through ctypes by the Python binding.
"""
module IPEPSB200

using ChainRulesCore

const lib = get(ENV, "IPEPS_B200_LIB", joinpath(@__DIR__, "..", "libipeps_b200.so"))

const IPEPS_CONV_ENERGY = Cint(0)
const IPEPS_CONV_SPECTRUM = Cint(1)
const IPEPS_CONV_ES = Cint(2)

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

"""Device-side counterpart of `CTMTensors` (ctm_tensor.jl:3-18); T is Float64
or ComplexF64 (the element type of A and of the environment)."""
mutable struct CTMTensorsB200{T<:Union{Float64,ComplexF64}}
    eng::Engine
    h::Ptr{Cvoid}
    A::Array{T,5}
    B::Union{Nothing,Array{ComplexF64,5}}
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

"""`CTMTensors(A, cfg)` (ctm_tensor.jl:63-69): Ad = conj(A), init_ctm1 on the
device.  `init=false` leaves C/T to `set_CT!` (a copy of another environment,
as optim_es.jl:127-131 starts every basis vector from the ground state's)."""
function CTMTensorsB200(A::AbstractArray{T,5}, cfg::Dict; eng::Engine=engine(),
                        init::Bool=true) where {T<:Union{Float64,ComplexF64}}
    D, d = size(A, 1), size(A, 5)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(eng.h, ccall((:ipeps_env_create, lib), Cint, (Ptr{Cvoid}, Cint, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
                       eng.h, D, d, get(cfg, "chi", 30), T <: Complex ? 1 : 0, r))
    ts = CTMTensorsB200{T}(eng, r[], Array{T,5}(A), nothing, Dict{String,Any}(cfg))
    finalizer(x -> ccall((:ipeps_env_destroy, lib), Cint, (Ptr{Cvoid},), x.h), ts)
    push_params!(ts)
    GC.@preserve ts begin
        check(eng.h, ccall((:ipeps_env_set_A, lib), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}),
                           ts.h, pointer(ts.A), C_NULL))
    end
    init && check(eng.h, ccall((:ipeps_env_init, lib), Cint, (Ptr{Cvoid},), ts.h))
    return ts
end

"""`ts.Cs[k]`, `ts.Es[k]` (k = 1..4) as host arrays."""
function get_CT(ts::CTMTensorsB200{T}, k::Integer) where {T}
    cd, ed = zeros(Int64, 2), zeros(Int64, 4)
    GC.@preserve cd ed begin
        check(ts.eng.h, ccall((:ipeps_env_get_CT, lib), Cint,
                              (Ptr{Cvoid}, Cint, Ptr{Cvoid}, Ptr{Int64}, Ptr{Cvoid}, Ptr{Int64}),
                              ts.h, k, C_NULL, cd, C_NULL, ed))
    end
    C, E = Array{T}(undef, cd...), Array{T}(undef, ed...)
    GC.@preserve C E cd ed begin
        check(ts.eng.h, ccall((:ipeps_env_get_CT, lib), Cint,
                              (Ptr{Cvoid}, Cint, Ptr{Cvoid}, Ptr{Int64}, Ptr{Cvoid}, Ptr{Int64}),
                              ts.h, k, pointer(C), cd, pointer(E), ed))
    end
    return C, E
end

function set_CT!(ts::CTMTensorsB200{T}, k::Integer, C::AbstractMatrix, E::AbstractArray) where {T}
    Cc, Ec = Array{T}(C), Array{T}(E)
    cd, ed = collect(Int64, size(Cc)), collect(Int64, size(Ec))
    GC.@preserve Cc Ec cd ed begin
        check(ts.eng.h, ccall((:ipeps_env_set_CT, lib), Cint,
                              (Ptr{Cvoid}, Cint, Ptr{Cvoid}, Ptr{Int64}, Ptr{Cvoid}, Ptr{Int64}),
                              ts.h, k, pointer(Cc), cd, pointer(Ec), ed))
    end
    return ts
end

"""`setproperties(ts, B=B, Bd=conj(B))` with `Params["px"], Params["py"]` in
radians (optim_es.jl:124-125, 171); clears the nested environment slots."""
function set_B!(ts::CTMTensorsB200, B::AbstractArray, px::Real, py::Real)
    ts.B = Array{ComplexF64,5}(reshape(B, size(ts.A)))
    ts.Params["px"], ts.Params["py"] = Float64(px), Float64(py)
    GC.@preserve ts begin
        check(ts.eng.h, ccall((:ipeps_nested_set_B, lib), Cint, (Ptr{Cvoid}, Ptr{ComplexF64}, Float64, Float64),
                              ts.h, ts.B, px, py))
    end
    return ts
end

hmat(h) = Matrix{ComplexF64}(h)

"""`run_ctm(ts; conv_fun)` (ctmrg.jl:1-55).  Pass the Hamiltonian pair `H` as
`conv_fun` for the energy criterion (get_gs_energy; with `es=true` the
nested criterion get_es_energy / get_all_norm of optim_es.jl:175), or
`nothing` for the spectrum criterion.  Returns (ts, last diff)."""
function run_ctm(ts::CTMTensorsB200; conv_fun=nothing, es::Bool=false)
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
                                  ts.h, es ? IPEPS_CONV_ES : IPEPS_CONV_ENERGY, Hh, Hv, size(Hh, 1), iters, diff, conv))
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

"""`get_es_energy(ts, H)` (evaluation.jl:31-45) of the nested environment."""
function get_es_energy(ts::CTMTensorsB200, H)
    Hh, Hv = hmat(H[1]), hmat(H[2])
    E = zeros(1)
    GC.@preserve Hh Hv E begin
        check(ts.eng.h, ccall((:ipeps_es_energy, lib), Cint,
                              (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{ComplexF64}, Cint, Ptr{Float64}),
                              ts.h, Hh, Hv, size(Hh, 1), E))
    end
    return E[1]
end

"""`get_all_norm(ts)` (evaluation.jl:61-77): (Nb, envB), envB the size of A."""
function get_all_norm(ts::CTMTensorsB200)
    nb = zeros(2)
    envB = Array{ComplexF64}(undef, size(ts.A))
    GC.@preserve nb envB begin
        check(ts.eng.h, ccall((:ipeps_all_norm, lib), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{ComplexF64}),
                              ts.h, nb, envB))
    end
    return complex(nb[1], nb[2]), envB
end

"""The pullback of `run_es` (optim_es.jl:184-188) w.r.t. B from the nested
environment held by ts: (E, gH), gH = dE/dRe B + i dE/dIm B (Zygote's
convention for a complex argument)."""
function es_energy_grad!(ts::CTMTensorsB200, H)
    Hh, Hv = hmat(H[1]), hmat(H[2])
    E = zeros(1)
    g = Array{ComplexF64}(undef, size(ts.A))
    GC.@preserve Hh Hv E g begin
        check(ts.eng.h, ccall((:ipeps_es_energy_grad, lib), Cint,
                              (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{ComplexF64}, Cint, Cint, Ptr{Float64}, Ptr{ComplexF64}),
                              ts.h, Hh, Hv, size(Hh, 1), get(ts.Params, "ad_max_iter", 4), E, g))
    end
    return E[1], g
end

"""
    get_es_grad(ts1, H, Bi)

`get_es_grad` (optim_es.jl:167-194) on the device: ts1 holds a copy of the
normalised ground-state environment (`init=false` + `set_CT!`) with
`Params["px"], Params["py"]` set; it is advanced in place (B set, nested
CTMRG to convergence, the pullback iterations).  Returns (gH, gN) as flat
vectors, gN = envB of get_all_norm after the pullback (optim_es.jl:189).
"""
function get_es_grad(ts1::CTMTensorsB200, H, Bi::AbstractVector)
    set_B!(ts1, Bi, get(ts1.Params, "px", 0.0), get(ts1.Params, "py", 0.0))
    run_ctm(ts1; conv_fun=H, es=true)
    _, gH = es_energy_grad!(ts1, H)
    _, gN = get_all_norm(ts1)
    return vec(gH), vec(gN)
end

"""The pullback of `run_gs` (optim_gs.jl:133-143) from the environment held by
ts (real A: the engine has no complex-A gradient)."""
function energy_grad!(ts::CTMTensorsB200{Float64}, H)
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

# ---- plaquette (2x2-cluster) observables of the h4 drivers and optim_wp

"""`ipeps_ctensor_t`: one complex column-major tensor of the plaquette MPO."""
struct CTensor
    data::Ptr{Float64}
    nd::Cint
    dims::NTuple{4,Int64}
end

"""The MPO [s1, s2, s3, s4] of `get_local_h` (src/model/local_h.jl:1-31) as C
tensors; keep the returned arrays alive (GC.@preserve) during the call."""
function mpo_tensors(H4)
    length(H4) == 4 || error("the plaquette Hamiltonian is the MPO [s1, s2, s3, s4]")
    arrs = [Array{ComplexF64}(h) for h in H4]
    cts = [CTensor(Ptr{Float64}(pointer(a)), Cint(ndims(a)),
                   ntuple(i -> i <= ndims(a) ? Int64(size(a, i)) : Int64(0), 4)) for a in arrs]
    return arrs, cts
end

"""`get_gs_energy_4x4(ts, H4)` (evaluation.jl:339-356); with `es=true`
`get_es_energy_4x4` (evaluation.jl:358-398, B set)."""
function get_energy_4x4(ts::CTMTensorsB200, H4; es::Bool=false)
    arrs, cts = mpo_tensors(H4)
    E = zeros(2)
    GC.@preserve arrs cts E begin
        check(ts.eng.h, ccall((:ipeps_energy_4x4, lib), Cint, (Ptr{Cvoid}, Ptr{CTensor}, Cint, Ptr{Float64}),
                              ts.h, cts, es ? 1 : 0, E))
    end
    return complex(E[1], E[2])
end

"""`run_ctm(ts; conv_fun = ts -> get_gs_energy_4x4(ts, H4))` (optim_gs_h4.jl);
`es=true`: the nested criterion of optim_es_h4.jl:139.  Returns (ts, last diff)."""
function run_ctm_4x4(ts::CTMTensorsB200, H4; es::Bool=false)
    push_params!(ts)
    arrs, cts = mpo_tensors(H4)
    iters, diff, conv = Ref{Cint}(0), Ref{Float64}(0), Ref{Cint}(0)
    GC.@preserve arrs cts begin
        check(ts.eng.h, ccall((:ipeps_ctm_run_4x4, lib), Cint,
                              (Ptr{Cvoid}, Ptr{CTensor}, Cint, Ref{Cint}, Ref{Float64}, Ref{Cint}),
                              ts.h, cts, es ? 1 : 0, iters, diff, conv))
    end
    conv[] == 0 && println("--------- Not Converged ----------")
    return ts, diff[]
end

"""The pullback of `run_gs_h4` (optim_gs_h4.jl:113-123) w.r.t. A (real A)."""
function energy_grad_4x4!(ts::CTMTensorsB200{Float64}, H4)
    arrs, cts = mpo_tensors(H4)
    E = zeros(1)
    g = similar(ts.A)
    GC.@preserve arrs cts E g begin
        check(ts.eng.h, ccall((:ipeps_energy_grad_4x4, lib), Cint,
                              (Ptr{Cvoid}, Ptr{CTensor}, Cint, Ptr{Float64}, Ptr{Float64}),
                              ts.h, cts, get(ts.Params, "ad_max_iter", 4), E, g))
    end
    return E[1], g
end

"""The pullback of `run_es_h4` w.r.t. B in `get_es_grad_h4` (optim_es_h4.jl:150-188)."""
function es_energy_grad_4x4!(ts::CTMTensorsB200, H4)
    arrs, cts = mpo_tensors(H4)
    E = zeros(1)
    g = Array{ComplexF64}(undef, size(ts.A))
    GC.@preserve arrs cts E g begin
        check(ts.eng.h, ccall((:ipeps_es_energy_grad_4x4, lib), Cint,
                              (Ptr{Cvoid}, Ptr{CTensor}, Cint, Ptr{Float64}, Ptr{ComplexF64}),
                              ts.h, cts, get(ts.Params, "ad_max_iter", 4), E, g))
    end
    return E[1], g
end

"""`get_wp_grad` (optim_wp.jl:195-238) in the environment held by ts (no
CTMRG): the plaquette operator wp4 (an MPO as for the energy) and the norm of
the cluster whose site `site` (Params["wp"], 1..4) holds B, the others A.
Returns (operator value, norm, gH, gN)."""
function get_wp_grad(ts::CTMTensorsB200, wp4, site::Integer, B::AbstractArray)
    arrs, cts = mpo_tensors(wp4)
    Bc = Array{ComplexF64}(reshape(B, size(ts.A)))
    vn = zeros(4)
    gH = Array{ComplexF64}(undef, size(ts.A))
    gN = Array{ComplexF64}(undef, size(ts.A))
    GC.@preserve arrs cts Bc vn gH gN begin
        check(ts.eng.h, ccall((:ipeps_wp_grad, lib), Cint,
                              (Ptr{Cvoid}, Ptr{CTensor}, Cint, Ptr{ComplexF64}, Ptr{Float64}, Ptr{ComplexF64},
                               Ptr{ComplexF64}),
                              ts.h, cts, site, Bc, vn, gH, gN))
    end
    return complex(vn[1], vn[2]), complex(vn[3], vn[4]), gH, gN
end

"""`run_gs_h4` of optim_gs_h4.jl:113-123 as one differentiable function
(converge with the plaquette energy, ad_max_iter iterations, the energy);
its rrule returns the hand-written adjoint for fg! (optim_gs_h4.jl:74)."""
function ctm_energy_h4(A::AbstractArray{Float64,5}, H4, cfg::Dict)
    ts = CTMTensorsB200(A, cfg)
    run_ctm_4x4(ts, H4)
    E, _ = energy_grad_4x4!(ts, H4)
    return E
end

function ChainRulesCore.rrule(::typeof(ctm_energy_h4), A::AbstractArray{Float64,5}, H4, cfg::Dict)
    ts = CTMTensorsB200(A, cfg)
    run_ctm_4x4(ts, H4)
    E, g = energy_grad_4x4!(ts, H4)
    ctm_energy_h4_pullback(dE) = (NoTangent(), unthunk(dE) .* g, NoTangent(), NoTangent())
    return E, ctm_energy_h4_pullback
end

end # module
