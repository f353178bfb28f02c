#=
SmoQCUDA.jl -- Julia binding of libsmoq_cuda.so (include/smoq_cuda.h).

Keeps the names and argument order of SmoQ.jl's utils/cpu functions and
dispatches them on `CuState`, a device-resident stand-in for
ψ::Vector{ComplexF64}.  Scripts switch from the CPU path to the GPU path by
constructing ψ as a CuState.  Qubits stay 1-based here; the C ABI takes k-1.
=#
module SmoQCUDA

export CuContext, CuState, apply_rx_psi!, apply_ry_psi!, apply_rz_psi!, apply_hadamard_psi!,
       apply_pauli_x_psi!, apply_pauli_y_psi!, apply_pauli_z_psi!, apply_s_psi!, apply_sdagger_psi!,
       apply_t_psi!, apply_tdagger_psi!, apply_cnot_psi!, apply_cz_psi!, apply_cry_psi!,
       apply_rxx_psi!, apply_ryy_psi!, apply_rzz_psi!, apply_ccz_psi!, apply_toffoli_psi!,
       apply_sigma_minus_psi!, apply_sigma_plus_psi!, apply_sigma_z!, population_excited_psi,
       expect_local, expect_corr, get_expectation_pauli_string, get_norm, normalize_state!,
       TrotterPlan, evolve_trotter_psi!, apply_fast_trotter_step_cpu!, energy_and_gradient,
       energy_and_gradient_jobs, lindblad_mcwf_batched!, apply_hamiltonian_bitwise!, sample_bitstrings,
       projective_measurement_all!, measure_z_single!, set_engine!, run_mcwf_simulation

const lib = joinpath(@__DIR__, "..", "lib", "libsmoq_cuda.so")
const SMOQ_C64 = Cint(0)
const SMOQ_C128 = Cint(1)

mutable struct CuContext
    h::Ptr{Cvoid}
    function CuContext(device::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:smoq_ctx_create, lib), Cint, (Cint, Ref{Ptr{Cvoid}}), device, r)
        st == 0 || error("smoq_ctx_create failed with status $st")
        c = new(r[])
        finalizer(c -> ccall((:smoq_ctx_destroy, lib), Cint, (Ptr{Cvoid},), c.h), c)
        c
    end
end

function check(st::Cint, ctx::CuContext)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:smoq_last_error, lib), Cstring, (Ptr{Cvoid},), ctx.h))
    throw(ErrorException(msg))
end

mutable struct CuState
    h::Ptr{Cvoid}
    ctx::CuContext
    N::Int
    batch::Int
    function CuState(ctx::CuContext, N::Integer; dtype=SMOQ_C128, batch::Integer=1, basis::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:smoq_state_create, lib), Cint, (Ptr{Cvoid}, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
                    ctx.h, N, dtype, batch, r), ctx)
        s = new(r[], ctx, N, batch)
        check(ccall((:smoq_state_set_basis, lib), Cint, (Ptr{Cvoid}, UInt64), s.h, basis), ctx)
        finalizer(s -> ccall((:smoq_state_destroy, lib), Cint, (Ptr{Cvoid},), s.h), s)
        s
    end
end

# ---------------------------------------------------------------- gates
for (jl, c) in ((:apply_rx_psi!, :smoq_apply_rx), (:apply_ry_psi!, :smoq_apply_ry), (:apply_rz_psi!, :smoq_apply_rz))
    @eval $jl(ψ::CuState, k::Int, θ::Float64, N::Int) =
        (check(ccall(($(QuoteNode(c)), lib), Cint, (Ptr{Cvoid}, Cint, Cdouble), ψ.h, k - 1, θ), ψ.ctx); ψ)
end
for (jl, c) in ((:apply_hadamard_psi!, :smoq_apply_h), (:apply_pauli_x_psi!, :smoq_apply_x),
                (:apply_pauli_y_psi!, :smoq_apply_y), (:apply_pauli_z_psi!, :smoq_apply_z),
                (:apply_sigma_z!, :smoq_apply_z), (:apply_s_psi!, :smoq_apply_s),
                (:apply_sdagger_psi!, :smoq_apply_sdg), (:apply_t_psi!, :smoq_apply_t),
                (:apply_tdagger_psi!, :smoq_apply_tdg), (:apply_sigma_minus_psi!, :smoq_apply_sigma_minus),
                (:apply_sigma_plus_psi!, :smoq_apply_sigma_plus))
    @eval $jl(ψ::CuState, k::Int, N::Int) =
        (check(ccall(($(QuoteNode(c)), lib), Cint, (Ptr{Cvoid}, Cint), ψ.h, k - 1), ψ.ctx); ψ)
end
for (jl, c) in ((:apply_cnot_psi!, :smoq_apply_cnot), (:apply_cz_psi!, :smoq_apply_cz))
    @eval $jl(ψ::CuState, a::Int, b::Int, N::Int) =
        (check(ccall(($(QuoteNode(c)), lib), Cint, (Ptr{Cvoid}, Cint, Cint), ψ.h, a - 1, b - 1), ψ.ctx); ψ)
end
for (jl, c) in ((:apply_cry_psi!, :smoq_apply_cry), (:apply_rxx_psi!, :smoq_apply_rxx),
                (:apply_ryy_psi!, :smoq_apply_ryy), (:apply_rzz_psi!, :smoq_apply_rzz))
    @eval $jl(ψ::CuState, a::Int, b::Int, θ::Float64, N::Int) =
        (check(ccall(($(QuoteNode(c)), lib), Cint, (Ptr{Cvoid}, Cint, Cint, Cdouble), ψ.h, a - 1, b - 1, θ), ψ.ctx); ψ)
end
for (jl, c) in ((:apply_ccz_psi!, :smoq_apply_ccz), (:apply_toffoli_psi!, :smoq_apply_toffoli))
    @eval $jl(ψ::CuState, a::Int, b::Int, t::Int, N::Int) =
        (check(ccall(($(QuoteNode(c)), lib), Cint, (Ptr{Cvoid}, Cint, Cint, Cint), ψ.h, a - 1, b - 1, t - 1), ψ.ctx); ψ)
end

# --------------------------------------------------------- observables
function _out(f, ψ::CuState, args...)
    out = Vector{Cdouble}(undef, ψ.batch)
    check(f(out), ψ.ctx)
    ψ.batch == 1 ? out[1] : out
end

function expect_local(ψ::CuState, k::Int, N::Int, pauli::Symbol)
    c = pauli === :z ? :smoq_expect_z : pauli === :x ? :smoq_expect_x : pauli === :y ? :smoq_expect_y :
        error("Unknown Pauli operator: $pauli. Use :x, :y, or :z")
    _out(o -> ccall((c, lib), Cint, (Ptr{Cvoid}, Cint, Ptr{Cdouble}), ψ.h, k - 1, o), ψ)
end

function expect_corr(ψ::CuState, i::Int, j::Int, N::Int, pair::Symbol)
    c = pair === :zz ? :smoq_expect_zz : pair === :xx ? :smoq_expect_xx : pair === :yy ? :smoq_expect_yy :
        error("Unknown Pauli pair: $pair. Use :zz, :xx, or :yy")
    _out(o -> ccall((c, lib), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}), ψ.h, i - 1, j - 1, o), ψ)
end

function get_expectation_pauli_string(ψ::CuState, ops::Vector{Symbol}, qubits::Vector{Int}, N::Int)
    isempty(ops) && return 1.0
    s = join(uppercase(String(o)) for o in ops)
    q = Cint.(qubits .- 1)
    _out(o -> ccall((:smoq_expect_pauli_string, lib), Cint, (Ptr{Cvoid}, Cint, Cstring, Ptr{Cint}, Ptr{Cdouble}),
                    ψ.h, length(q), s, q, o), ψ)
end

population_excited_psi(ψ::CuState, k::Int, N::Int) =
    _out(o -> ccall((:smoq_population_excited, lib), Cint, (Ptr{Cvoid}, Cint, Ptr{Cdouble}), ψ.h, k - 1, o), ψ)
get_norm(ψ::CuState) = sqrt.(_out(o -> ccall((:smoq_norm2, lib), Cint, (Ptr{Cvoid}, Ptr{Cdouble}), ψ.h, o), ψ))
normalize_state!(ψ::CuState) = (check(ccall((:smoq_normalize, lib), Cint, (Ptr{Cvoid},), ψ.h), ψ.ctx); ψ)

# -------------------------------------------------------------- Trotter
struct CTrotterGate
    nq::Int32
    q1::Int32
    q2::Int32
    pad::Int32
    U::NTuple{32,Float64}
end

mutable struct TrotterPlan
    h::Ptr{Cvoid}
    ctx::CuContext
end

"gates: Vector of (indices::Vector{Int}, U::Matrix{ComplexF64}) as in FastTrotterGate"
function TrotterPlan(ctx::CuContext, N::Int, gates; order::Int=1, dtype=SMOQ_C128)
    cg = map(gates) do (idx, U)
        u = reinterpret(Float64, vec(ComplexF64.(U)))     # column-major, interleaved
        pad = ntuple(i -> i <= length(u) ? u[i] : 0.0, 32)
        CTrotterGate(length(idx), idx[1] - 1, length(idx) > 1 ? idx[2] - 1 : 0, 0, pad)
    end
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:smoq_trotter_plan_create, lib), Cint,
                (Ptr{Cvoid}, Cint, Cint, Ptr{CTrotterGate}, Cint, Cint, Ref{Ptr{Cvoid}}),
                ctx.h, N, dtype, cg, length(cg), order, r), ctx)
    p = TrotterPlan(r[], ctx)
    finalizer(p -> ccall((:smoq_plan_destroy, lib), Cint, (Ptr{Cvoid},), p.h), p)
    p
end

# evolve_trotter_psi_cpu!(psi, gates, N, n_substeps) -- Trotter.jl:250
evolve_trotter_psi!(ψ::CuState, plan::TrotterPlan, N::Int, n::Int=1) =
    (check(ccall((:smoq_trotter_step, lib), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint), plan.h, ψ.h, n), ψ.ctx); ψ)
# apply_fast_trotter_step_cpu!(psi, gates, N) -- Trotter.jl:150
apply_fast_trotter_step_cpu!(ψ::CuState, plan::TrotterPlan, N::Int) = evolve_trotter_psi!(ψ, plan, N, 1)

# ------------------------------------------------ VQE energy + adjoint grad
struct CPauliTerm
    coef::Float64
    xmask::UInt64
    zmask::UInt64
end

struct COp
    type::Int32
    q::NTuple{3,Int32}
    param::Int32
    pad::Int32
    angle::Float64
    U::NTuple{32,Float64}
end

"θ: n_params × batch; returns (energies, grads::Matrix)"
function energy_and_gradient(ctx::CuContext, N::Int, ops::Vector{COp}, n_params::Int,
                             H::Vector{CPauliTerm}, θ::Matrix{Float64}; dtype=SMOQ_C128)
    B = size(θ, 2)
    E = Vector{Float64}(undef, B)
    G = Matrix{Float64}(undef, n_params, B)
    check(ccall((:smoq_energy_grad, lib), Cint,
                (Ptr{Cvoid}, Cint, Cint, Ptr{COp}, Cint, Cint, Ptr{CPauliTerm}, Cint, Cint,
                 Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                ctx.h, N, dtype, ops, length(ops), n_params, H, length(H), B, θ, E, G), ctx)
    E, G
end

# ChainRulesCore (Manifest.toml:254, 1.26.0) -- the adjoint behind an rrule:
#   function ChainRulesCore.rrule(::typeof(vqe_energy), θ)
#       E, G = energy_and_gradient(ctx, N, ops, length(θ), H, reshape(θ, :, 1))
#       return E[1], Δ -> (NoTangent(), Δ .* G[:, 1])
#   end

# ------------------------------------------------ many circuits (C4b)
struct CVqeJob
    N::Cint
    ops::Ptr{COp}
    n::Cint
    n_params::Cint
    H::Ptr{CPauliTerm}
    nterms::Cint
    theta::Ptr{Float64}
    energy::Ptr{Float64}
    grad::Ptr{Float64}
end

"jobs: Vector of (N, ops::Vector{COp}, n_params, H::Vector{CPauliTerm}, θ::Vector{Float64});
returns (energies, grads) -- each circuit its own size and Hamiltonian"
function energy_and_gradient_jobs(ctx::CuContext, jobs; dtype=SMOQ_C128)
    E = Vector{Float64}(undef, length(jobs))
    G = [Vector{Float64}(undef, j[3]) for j in jobs]
    GC.@preserve jobs E G begin
        cj = [CVqeJob(j[1], pointer(j[2]), length(j[2]), j[3], pointer(j[4]), length(j[4]), pointer(j[5]),
                      pointer(E, i), pointer(G[i])) for (i, j) in enumerate(jobs)]
        check(ccall((:smoq_energy_grad_jobs, lib), Cint, (Ptr{Cvoid}, Cint, Ptr{CVqeJob}, Cint),
                    ctx.h, dtype, cj, length(cj)), ctx)
    end
    E, G
end

# ------------------------------------------------------------------ MCWF
struct CJumpOp
    type::Int32       # 0 sigma-, 1 sigma+, 2 sigma_z, 3 sigma_x
    qubit::Int32      # 0-based
    gamma::Float64
end

"evolve_mcwf_batched_trotter! (MonteCarloWaveFunction.jl:412) on the GPU: every state
of ψ (batch = trajectories) evolves under `plan` (order 1) and `jumps`; returns the
trajectory means of <Z_i> and <Z_i Z_{i+1}> every `record_every` steps and the jump counts."
function lindblad_mcwf_batched!(ψ::CuState, plan::TrotterPlan, jumps::Vector{CJumpOp}, dt::Float64,
                                seed::UInt64, steps::Int, record_every::Int)
    nrec = steps ÷ record_every + 1
    z = Matrix{Float64}(undef, ψ.N, nrec)
    zz = Matrix{Float64}(undef, ψ.N - 1, nrec)
    nj = Vector{Cint}(undef, ψ.batch)
    check(ccall((:smoq_mcwf_run, lib), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{CJumpOp}, Cint, Cdouble, UInt64, UInt64, Cint, Cint,
                 Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Cint}),
                plan.h, ψ.h, jumps, length(jumps), dt, seed, 0, steps, record_every, z, zz, C_NULL, C_NULL, nj),
          ψ.ctx)
    z, zz, nj
end

# ------------------------------------------------ H ψ, sampling, measurement
"apply_hamiltonian_bitwise!(ψ_out, ψ_in, params) -- Chebyshev.jl:55, for a Pauli sum; returns <ψ_in|H|ψ_in>"
function apply_hamiltonian_bitwise!(ψout::CuState, ψin::CuState, H::Vector{CPauliTerm})
    e = Vector{Float64}(undef, ψin.batch)
    check(ccall((:smoq_apply_pauli_sum, lib), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{CPauliTerm}, Cint, Ptr{Float64}),
                ψin.h, ψout.h, H, length(H), e), ψin.ctx)
    ψin.batch == 1 ? e[1] : e
end

"Born shots (0-based basis indices), the benchmark's cumsum + searchsortedfirst loop"
function sample_bitstrings(ψ::CuState, nshots::Int; seed::UInt64=UInt64(42), stream::UInt64=UInt64(0))
    out = Matrix{Int64}(undef, nshots, ψ.batch)
    check(ccall((:smoq_sample, lib), Cint, (Ptr{Cvoid}, Clonglong, Culonglong, Culonglong, Ptr{Int64}),
                ψ.h, nshots, seed, stream, out), ψ.ctx)
    out
end

"projective_measurement_all!(ψ, N) -- Measurements.jl:484: (bitstring, ψ collapsed)"
function projective_measurement_all!(ψ::CuState, N::Int; seed::UInt64=UInt64(42), stream::UInt64=UInt64(0))
    o = Vector{Int64}(undef, ψ.batch)
    check(ccall((:smoq_measure_all, lib), Cint, (Ptr{Cvoid}, Culonglong, Culonglong, Ptr{Int64}),
                ψ.h, seed, stream, o), ψ.ctx)
    [(o[1] >> (k - 1)) & 1 for k in 1:N], ψ
end

"_measure_z_single!(ψ, k, N) -- Measurements.jl:224: outcome 0/1, ψ collapsed"
function measure_z_single!(ψ::CuState, k::Int, N::Int; seed::UInt64=UInt64(42), stream::UInt64=UInt64(0))
    o = Vector{Cint}(undef, ψ.batch)
    check(ccall((:smoq_measure_qubit, lib), Cint, (Ptr{Cvoid}, Cint, Culonglong, Culonglong, Ptr{Cint}),
                ψ.h, k - 1, seed, stream, o), ψ.ctx)
    ψ.batch == 1 ? Int(o[1]) : Int.(o)
end

struct CQrcParams
    L::Int32; n_substeps::Int32; encoding::Int32; reset::Int32
    seed::UInt64; traj_offset::UInt64
end

"""run_mcwf_simulation(psi0, H_params, gates, padded_u, L, n_rails, T, n_traj, :trotter_cpu,
T_evol, encoding, reset_type, n_substeps) -- the bitwise QRC loop
(cpuQRCSimulationMonteCarloWaveFunction.jl:531) on the GPU; `gates` is a TrotterPlan on
N = 2L qubits.  Returns X (T x n_ops), the trajectory mean of the ladder features."""
function run_mcwf_simulation(psi0, H_params, gates::TrotterPlan, padded_u::Vector{Float64}, L::Int,
                             n_rails::Int, T::Int, n_traj::Int, integrator_type::Symbol, T_evol::Float64,
                             encoding::Symbol, reset_type::Symbol, n_substeps::Int=5;
                             seed::UInt64=UInt64(1234), traj_offset::UInt64=UInt64(0))
    integrator_type == :trotter_cpu || error("Unsupported integrator: $integrator_type. Supported: :trotter_cpu")
    n_rails == 2 || error("the QRC reset reshapes the state as 2^L x 2^L: n_rails must be 2")
    enc = encoding == :broadcast ? 1 : 0
    rst = reset_type in (:traceout_rail_1, :protocol1) ? 1 : reset_type in (:traceout_rail_2, :protocol2) ? 2 :
          error("Unknown protocol: $reset_type. Use :traceout_rail_1 or :traceout_rail_2")
    p = Ref(CQrcParams(L, n_substeps, enc, rst, seed, traj_offset))
    n_ops = 3 * 2L + 3 * (L - 1) * 2 + 3 * L
    X = Vector{Float64}(undef, T * n_ops)
    p0 = psi0 === nothing ? C_NULL : reinterpret(Float64, Vector{ComplexF64}(psi0))
    check(ccall((:smoq_qrc_run, lib), Cint,
                (Ptr{Cvoid}, Ref{CQrcParams}, Ptr{Float64}, Ptr{Float64}, Cint, Int64, Ptr{Float64}, Ptr{Float64}),
                gates.h, p, p0, padded_u, T, n_traj, X, C_NULL), gates.ctx)
    permutedims(reshape(X, n_ops, T))   # X[k, f], as the reference's Matrix (T x n_ops)
end

"fused-pass engine: -1 auto (default), 0 shared-memory sweeps, 1 register tiles, 2 stage
sweeps, 3 compiled pass kernels"
set_engine!(ctx::CuContext, e::Integer) =
    check(ccall((:smoq_ctx_set_option, lib), Cint, (Ptr{Cvoid}, Cint, Clonglong), ctx.h, 7, e), ctx)

end # module
