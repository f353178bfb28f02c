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
       projective_measurement_all!, measure_z_single!, set_engine!, set_option!, run_mcwf_simulation,
       apply_gate!, apply_2qubit_gate!, apply_one_qubit_gate_bitwise_cpu!, apply_two_qubit_gate_bitwise_cpu!,
       apply_circuit!, apply_channel_dephasing!, apply_channel_depolarizing!, apply_channel_amplitude_damping!,
       apply_channel_bit_flip!, apply_channel_phase_flip!, projective_measurement!, reset_state!,
       VQECost, calculate_gradients, apply_H_xxz!, apply_H_ising!, energy_and_gradient_noisy

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

# host <-> device: CuState(ctx, psi::Vector{ComplexF64}) uploads, Vector(psi) downloads
function CuState(ctx::CuContext, ψ::Vector{ComplexF64})
    N = trailing_zeros(length(ψ))
    length(ψ) == 1 << N || error("State dimension mismatch")
    s = CuState(ctx, N)
    check(ccall((:smoq_state_upload, lib), Cint, (Ptr{Cvoid}, Ptr{ComplexF64}, Csize_t), s.h, ψ, sizeof(ψ)), ctx)
    s
end
function Base.Vector(ψ::CuState)
    out = Vector{ComplexF64}(undef, ψ.batch << ψ.N)
    check(ccall((:smoq_state_download, lib), Cint, (Ptr{Cvoid}, Ptr{ComplexF64}, Csize_t), ψ.h, out, sizeof(out)),
          ψ.ctx)
    out
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

# generic matrices.  apply_gate!(psi, U, qubit, N) (RandomUnitaries.jl:230) and
# apply_one_qubit_gate_bitwise_cpu!(psi, U, qubit, N) (Trotter.jl:77): U a 2x2 Matrix{ComplexF64};
# apply_2qubit_gate! (RandomUnitaries.jl:317) conjugates U by SWAP when q1 > q2 (convention 1);
# apply_two_qubit_gate_bitwise_cpu! (Trotter.jl:107) swaps the qubits and keeps U (convention 0)
function _u1(ψ::CuState, U::Matrix{ComplexF64}, q::Int)
    size(U) == (2, 2) || error("U must be 2x2")
    check(ccall((:smoq_apply_u1, lib), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}), ψ.h, q - 1, U), ψ.ctx)
    ψ
end
function _u2(ψ::CuState, U::Matrix{ComplexF64}, q1::Int, q2::Int, convention::Int)
    size(U) == (4, 4) || error("U must be 4x4")
    check(ccall((:smoq_apply_u2, lib), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{ComplexF64}, Cint),
                ψ.h, q1 - 1, q2 - 1, U, convention), ψ.ctx)
    ψ
end
apply_gate!(ψ::CuState, U::Matrix{ComplexF64}, qubit::Int, N::Int) = _u1(ψ, U, qubit)
apply_one_qubit_gate_bitwise_cpu!(ψ::CuState, U::Matrix{ComplexF64}, qubit::Int, N::Int) = _u1(ψ, U, qubit)
apply_2qubit_gate!(ψ::CuState, U::Matrix{ComplexF64}, q1::Int, q2::Int, N::Int) = _u2(ψ, U, q1, q2, 1)
apply_two_qubit_gate_bitwise_cpu!(ψ::CuState, U::Matrix{ComplexF64}, q1::Int, q2::Int, N::Int) = _u2(ψ, U, q1, q2, 0)

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
    if_outcome::Int32
    angle::Float64
    U::NTuple{32,Float64}
end

# the CircuitOperation symbols (cpuVariationalQuantumCircuitBuilder.jl:82-94) -> smoq_op types
const GATE_CODE = Dict(:rx => 0, :ry => 1, :rz => 2, :h => 3, :x => 4, :y => 5, :z => 6, :s => 7, :sdg => 8,
                       :t => 9, :tdg => 10, :cz => 11, :cnot => 12, :cx => 12, :rxx => 13, :ryy => 14, :rzz => 15,
                       :cry => 16, :ccz => 17, :toffoli => 18)
const NOISE_CODE = Dict(:depolarizing => 32, :amplitude_damping => 33, :dephasing => 34, :bit_flip => 35,
                        :phase_flip => 36, :phase_damping => 37, :thermal_relaxation => 38)
const MEASURE_CODE = Dict(:measure_z => 48, :measure_x => 49, :measure_y => 50, :measure => 48)
const OTHER_CODE = Dict(:reset => 51, :trace_out => 52, :lindblad_step => 53)
const RESET_TARGET = Dict(:zero => 0, :one => 1, :plus => 2, :minus => 3)
const NOU = ntuple(_ -> 0.0, 32)

"the reference's CircuitOperation list (any object with its fields) as smoq_op records:
one record per gate, one per qubit of a noise / measure / reset op"
function c_ops(operations)
    out = COp[]
    for op in operations
        t = op.type
        if haskey(GATE_CODE, t)
            q = ntuple(k -> k <= length(op.qubits) ? Int32(op.qubits[k] - 1) : Int32(0), 3)
            push!(out, COp(GATE_CODE[t], q, op.param_idx > 0 ? op.param_idx - 1 : -1, op.if_outcome,
                           op.fixed_angle, NOU))
        else
            code = get(NOISE_CODE, t, get(MEASURE_CODE, t, get(OTHER_CODE, t, -1)))
            code < 0 && error("Unknown operation type: $t")
            for q in op.qubits
                q2 = t === :reset ? RESET_TARGET[op.target_state] : 0
                push!(out, COp(code, (Int32(q - 1), Int32(q2), Int32(0)), -1, op.if_outcome, op.p, NOU))
            end
        end
    end
    out
end
n_measurements(operations) = sum((length(op.qubits) for op in operations if haskey(MEASURE_CODE, op.type)); init=0)

"""apply_circuit!(ψ::CuState, circuit, θ) -- cpuVariationalQuantumCircuitExecutor.jl:95.
`circuit` is the reference's ParameterizedCircuit (fields N, operations).  Gate-only
circuits run as fused tile passes; circuits with noise, measurements, resets or
if_outcome conditions run every state of ψ as one trajectory (Philox draws, key seed,
counter (op index, 0x80000000, traj_offset + b)).  Returns (state = ψ, outcomes), the
fields of the reference's CircuitResult; outcomes is a Vector (one trajectory) or a
Matrix (outcome, trajectory)."""
function apply_circuit!(ψ::CuState, circuit, θ::Vector{Float64}; seed::UInt64=UInt64(1234),
                        traj_offset::UInt64=UInt64(0))
    ψ.N == circuit.N || error("State dimension mismatch")
    length(θ) >= circuit.n_params || error("Not enough parameters")
    ops = c_ops(circuit.operations)
    plain = all(op -> haskey(GATE_CODE, op.type) && op.if_outcome == 0, circuit.operations)
    if plain
        check(ccall((:smoq_apply_sequence, lib), Cint, (Ptr{Cvoid}, Ptr{COp}, Cint, Ptr{Float64}),
                    ψ.h, ops, length(ops), θ), ψ.ctx)
        return (state = ψ, outcomes = Int[])
    end
    nm = n_measurements(circuit.operations)
    out = Matrix{Int32}(undef, max(nm, 1), ψ.batch)
    check(ccall((:smoq_apply_circuit_mcwf, lib), Cint,
                (Ptr{Cvoid}, Ptr{COp}, Cint, Ptr{Float64}, UInt64, UInt64, Ptr{Int32}),
                ψ.h, ops, length(ops), θ, seed, traj_offset, out), ψ.ctx)
    o = Int.(out[1:nm, :])
    (state = ψ, outcomes = ψ.batch == 1 ? vec(o) : o)
end

# the public channels on pure states (cpuQuantumChannelKrausOperators.jl:426-556):
# one stochastic unravelling per state of ψ
for (jl, t) in ((:apply_channel_dephasing!, :dephasing), (:apply_channel_depolarizing!, :depolarizing),
                (:apply_channel_amplitude_damping!, :amplitude_damping), (:apply_channel_bit_flip!, :bit_flip),
                (:apply_channel_phase_flip!, :phase_flip))
    @eval function $jl(ψ::CuState, p::Float64, qubits::Vector{Int}, N::Int; seed::UInt64=UInt64(1234),
                       traj_offset::UInt64=UInt64(0))
        ops = [COp($(NOISE_CODE[t]), (Int32(q - 1), Int32(0), Int32(0)), -1, 0, p, NOU) for q in qubits]
        check(ccall((:smoq_apply_circuit_mcwf, lib), Cint,
                    (Ptr{Cvoid}, Ptr{COp}, Cint, Ptr{Float64}, UInt64, UInt64, Ptr{Int32}),
                    ψ.h, ops, length(ops), C_NULL, seed, traj_offset, C_NULL), ψ.ctx)
        ψ
    end
end

"projective_measurement!(ψ, qubits, basis, N) -- cpuQuantumStateMeasurements.jl:319: (outcomes, ψ)"
function projective_measurement!(ψ::CuState, qubits::Vector{Int}, basis::Symbol, N::Int; seed::UInt64=UInt64(1234),
                                 traj_offset::UInt64=UInt64(0))
    code = get(MEASURE_CODE, Symbol("measure_", basis), -1)
    code < 0 && error("Unknown basis: $basis. Use :z, :x, :y, or provide Vector/Matrix.")
    ops = [COp(code, (Int32(q - 1), Int32(0), Int32(0)), -1, 0, 0.0, NOU) for q in qubits]
    out = Matrix{Int32}(undef, length(qubits), ψ.batch)
    check(ccall((:smoq_apply_circuit_mcwf, lib), Cint,
                (Ptr{Cvoid}, Ptr{COp}, Cint, Ptr{Float64}, UInt64, UInt64, Ptr{Int32}),
                ψ.h, ops, length(ops), C_NULL, seed, traj_offset, out), ψ.ctx)
    (ψ.batch == 1 ? Int.(vec(out)) : Int.(out)), ψ
end

"reset_state!(ψ, qubits, target_states, N) -- cpuQuantumStateMeasurements.jl:555"
function reset_state!(ψ::CuState, qubits::Vector{Int}, targets, N::Int; seed::UInt64=UInt64(1234),
                      traj_offset::UInt64=UInt64(0))
    ts = targets isa Symbol ? fill(targets, length(qubits)) : targets
    length(ts) == length(qubits) || error("Must specify target for each qubit")
    ops = [COp(51, (Int32(q - 1), Int32(RESET_TARGET[t]), Int32(0)), -1, 0, 0.0, NOU) for (q, t) in zip(qubits, ts)]
    check(ccall((:smoq_apply_circuit_mcwf, lib), Cint,
                (Ptr{Cvoid}, Ptr{COp}, Cint, Ptr{Float64}, UInt64, UInt64, Ptr{Int32}),
                ψ.h, ops, length(ops), C_NULL, seed, traj_offset, C_NULL), ψ.ctx)
    ψ
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

"""VQECost(ctx, circuit, H; dtype): the VQE cost θ -> <0|U(θ)^dag H U(θ)|0> of the
reference's cost closures (scripts_variational_quantum_circuits/demo_vqe_dm_vs_mcwf.jl:189-202)
as a callable object; H is a Vector of (coef, Dict(qubit => :X/:Y/:Z)) terms."""
struct VQECost
    ctx::CuContext
    N::Int
    ops::Vector{COp}
    n_params::Int
    H::Vector{CPauliTerm}
    dtype::Cint
end
function pauli_terms(H)
    map(H) do (c, letters)
        x = UInt64(0); z = UInt64(0)
        for (q, P) in letters
            b = UInt64(1) << (q - 1)
            (P === :X || P === :Y) && (x |= b)
            (P === :Z || P === :Y) && (z |= b)
        end
        CPauliTerm(c, x, z)
    end
end
VQECost(ctx::CuContext, circuit, H; dtype=SMOQ_C128) =
    VQECost(ctx, circuit.N, c_ops(circuit.operations), circuit.n_params, pauli_terms(H), dtype)
(c::VQECost)(θ::AbstractVector{<:Real}) =
    energy_and_gradient(c.ctx, c.N, c.ops, c.n_params, c.H, reshape(Float64.(θ), :, 1); dtype=c.dtype)[1][1]

"""calculate_gradients(cost::VQECost, θ) -- cpuVariationalQuantumCircuitGradients.jl:88 with the
adjoint method as the backend (one forward sweep, one uncompute sweep) instead of Enzyme or the
parameter shift; returns the gradient vector."""
calculate_gradients(c::VQECost, θ::Vector{Float64}) =
    vec(energy_and_gradient(c.ctx, c.N, c.ops, c.n_params, c.H, reshape(θ, :, 1); dtype=c.dtype)[2])

# ChainRulesCore.rrule for the cost: reverse-mode AD (Zygote, a dependency of the reference's
# Project.toml, which loads ChainRulesCore 1.26.0, Manifest.toml:254) calls the adjoint kernels
# instead of differentiating through the gate loops.
import Zygote
const ChainRulesCore = Zygote.ChainRulesCore
function ChainRulesCore.rrule(c::VQECost, θ::AbstractVector{<:Real})
    E, G = energy_and_gradient(c.ctx, c.N, c.ops, c.n_params, c.H, reshape(Float64.(θ), :, 1); dtype=c.dtype)
    vqe_cost_pullback(ΔE) = (ChainRulesCore.NoTangent(), ΔE .* G[:, 1])
    return E[1], vqe_cost_pullback
end

"""energy_and_gradient_noisy(ctx, circuit, H, θ; seed, traj_offset, n_traj, checkpoint_every)
-- the path-wise adjoint gradient of a noisy circuit along fixed trajectories
(smoq_energy_grad_mcwf): returns (energies[n_traj], grads[n_params, n_traj])."""
function energy_and_gradient_noisy(ctx::CuContext, circuit, H, θ::Vector{Float64}; seed::UInt64=UInt64(1234),
                                   traj_offset::UInt64=UInt64(0), n_traj::Int=1, checkpoint_every::Int=1,
                                   dtype=SMOQ_C128)
    ops = c_ops(circuit.operations)
    terms = pauli_terms(H)
    E = Vector{Float64}(undef, n_traj)
    G = Matrix{Float64}(undef, max(circuit.n_params, 1), n_traj)
    check(ccall((:smoq_energy_grad_mcwf, lib), Cint,
                (Ptr{Cvoid}, Cint, Cint, Ptr{COp}, Cint, Cint, Ptr{CPauliTerm}, Cint, Ptr{Float64}, UInt64, UInt64,
                 Cint, Cint, Ptr{Float64}, Ptr{Float64}),
                ctx.h, circuit.N, dtype, ops, length(ops), circuit.n_params, terms, length(terms), θ, seed,
                traj_offset, n_traj, checkpoint_every, E, G), ctx)
    E, G[1:circuit.n_params, :]
end

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
"""apply_hamiltonian_bitwise!(ψ_out, ψ_in, params::HamiltonianParams) -- Chebyshev.jl:55:
ψ_out = H ψ_in for the reference's HamiltonianParams (fields x_bonds, y_bonds of CouplingTerm
(i, j, Jxx, Jyy, Jzz) and fields of FieldTerm (idx, hx, hy, hz), 1-based sites)"""
function apply_hamiltonian_bitwise!(ψout::CuState, ψin::CuState, params)
    rows(bs) = isempty(bs) ? Float64[] : reduce(vcat, [[b.i - 1, b.j - 1, b.Jxx, b.Jyy, b.Jzz] for b in bs])
    xb = rows(params.x_bonds); yb = rows(params.y_bonds)
    fb = isempty(params.fields) ? Float64[] : reduce(vcat, [[f.idx - 1, f.hx, f.hy, f.hz] for f in params.fields])
    check(ccall((:smoq_apply_hamiltonian_bitwise, lib), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Cint, Ptr{Float64}, Cint, Ptr{Float64}, Cint),
                ψout.h, ψin.h, xb, length(params.x_bonds), yb, length(params.y_bonds), fb, length(params.fields)),
          ψin.ctx)
    ψout
end
"apply_H_xxz!(ψ, out, N, Jx, Jy, Jz, h) -- cpuQuantumStateLanczos.jl:157"
apply_H_xxz!(ψ::CuState, out::CuState, N::Int, Jx::Float64, Jy::Float64, Jz::Float64, h::Float64) =
    (check(ccall((:smoq_apply_h_xxz, lib), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Cdouble),
                 ψ.h, out.h, Jx, Jy, Jz, h), ψ.ctx); out)
"apply_H_ising!(ψ, out, N, J, h) -- cpuQuantumStateLanczos.jl:220"
apply_H_ising!(ψ::CuState, out::CuState, N::Int, J::Float64, h::Float64) = apply_H_xxz!(ψ, out, N, 0.0, 0.0, J, h)

"apply_hamiltonian_bitwise! for a Pauli sum; returns <ψ_in|H|ψ_in>"
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

"fused-pass engine: -1 auto (default), 0 shared-memory sweeps, 2 stage sweeps, 3 compiled
pass kernels"
set_engine!(ctx::CuContext, e::Integer) =
    check(ccall((:smoq_ctx_set_option, lib), Cint, (Ptr{Cvoid}, Cint, Clonglong), ctx.h, 7, e), ctx)

# the context options of smoq_cuda.h (SMOQ_OPT_*) by name
const OPTIONS = Dict(:tile_bits_c64 => 1, :tile_bits_c128 => 2, :low_bits_c64 => 3, :low_bits_c128 => 4,
                     :use_graphs => 5, :kernel_timing => 6, :engine => 7, :jit_buffers => 8, :jit_groups => 10,
                     :vqe_resident => 12, :autotune => 13, :fusion_depth => 14)

"set a context option by name, e.g. `set_option!(ctx, :autotune, 2)` (tune the compiled
pass kernels' variants only, keeping the geometry the tile/low-bits/fusion-depth options
set; 1 = also time the candidate geometries, 0 = off)"
function set_option!(ctx::CuContext, name::Symbol, value::Integer)
    haskey(OPTIONS, name) || error("Unknown option: $name")
    check(ccall((:smoq_ctx_set_option, lib), Cint, (Ptr{Cvoid}, Cint, Clonglong), ctx.h, OPTIONS[name], value), ctx)
end

end # module
