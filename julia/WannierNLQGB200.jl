# WannierNLQGB200.jl - ccall binding of libwnlqg_b200.so for WannierNLQG (not executed in this
# repository: Julia is not installed in its build image).  A maintainer includes this file in
# WannierNLQG's Runtime and selects it with `fourier_backend = "b200"`.
module WannierNLQGB200

const LIB = get(ENV, "WNLQG_B200_LIB", joinpath(@__DIR__, "..", "wanniernlqg_b200", "libwnlqg_b200.so"))

const SHIFT_CURRENT = Int32(1)
const INJECTION_CURRENT = Int32(2)
const BERRY_CURVATURE = Int32(3)
const QUANTUM_METRIC = Int32(4)
const INTRINSIC_AHC = Int32(5)
const BERRY_DIPOLE = Int32(6)
const SECOND_HARMONIC = Int32(7)
const JERK_CURRENT = Int32(8)
const LINEAR_TRANSPORT_BERRY = Int32(9)
const BERRY_DIPOLE_SEA = Int32(10)            # Fermi-sea D^{abc}, finite-difference geometry

struct ModelDesc
    num_orbitals::Int64
    num_r_vectors::Int64
    lattice::Ptr{Float64}
    r_vectors::Ptr{Int64}
    r_degeneracies::Ptr{Int64}
    hamiltonian_r::Ptr{ComplexF64}
    position_r::Ptr{ComplexF64}
    overlap_r::Ptr{ComplexF64}
end

struct ResponseRequest
    kind::Int32
    num_components::Int32
    components::NTuple{324, Int32}     # [81][4], 0-based axes, a fastest
end

struct TaskDesc
    num_responses::Int32
    responses::NTuple{8, ResponseRequest}
    fermi_energy::Float64
    temperature::Float64
    broadening_type::Int32             # 0 Gaussian, 1 Lorentzian
    broadening::Float64
    transition_window_factor::Float64
    denominator_regularization::Float64
    degeneracy_threshold::Float64
    num_photon_energies::Int64
    photon_energies::Ptr{Float64}
    num_fermi_energies::Int64
    fermi_energies::Ptr{Float64}
    precision::Int32                   # 0 FP64, 1 mixed
    fermi_surface_broadening::Float64
    shg_low_frequency_broadening::Float64      # cfg.shg_low_frequency_broadening
    shg_intermediate_regularization::Float64   # cfg.shg_intermediate_regularization (0: denominator_regularization)
    shg_eta_correction::Int32                  # cfg.shg_eta_correction
    band_window_size::Int32                    # cfg.band_window_size (-1: all bands)
    use_band_selection::Int32                  # 1: cfg.band_selection = (conduction, valence) is set
    valence_bands::NTuple{4, UInt32}           # bit (n - 1) for valence band n
    conduction_bands::NTuple{4, UInt32}        # bit (m - 1) for conduction band m
    wannier_center_convention::Int32           # 0: CONVENTION_II, 1: CONVENTION_I
    spectral_gap_tolerance::Float64            # cfg.spectral_gap_tolerance (reference default 1e-10)
    linear_transport_gamma_inter::Float64      # cfg.gamma_inter_ev of the linear transport Berry channel
    finite_difference_step::Float64            # cfg.finite_difference_step (1/Angstrom, reference default 1e-4)
    derivative_backend::Int32                  # cfg.derivative_backend: 0 :finite_difference, 1 :analytic
end

function check(status)
    status == 0 && return nothing
    buf = Vector{UInt8}(undef, 4096)
    ccall((:wnlqg_b200_last_error, LIB), Cint, (Ptr{UInt8}, Csize_t), buf, length(buf))
    msg = unsafe_string(pointer(buf))
    status == 1 ? throw(ArgumentError(msg)) : status == 2 ? throw(DimensionMismatch(msg)) : error(msg)
end

"""Device-resident copy of a TightBindingModel (arrays are passed without copies)."""
function model_create(model; device::Integer = 0)
    desc = ModelDesc(model.num_orbitals, model.num_r_vectors, pointer(model.lattice),
                     pointer(model.r_vectors), pointer(model.r_degeneracies),
                     pointer(model.hamiltonian_r), pointer(model.position_r), C_NULL)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve model begin
        check(ccall((:wnlqg_b200_model_create, LIB), Cint, (Ref{ModelDesc}, Int32, Ref{Ptr{Cvoid}}),
                    desc, Int32(device), out))
    end
    return out[]
end

function plan_create(handle::Ptr{Cvoid}, task::TaskDesc; max_batch::Integer = 0)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:wnlqg_b200_plan_create, LIB), Cint, (Ptr{Cvoid}, Ref{TaskDesc}, Int64, Ref{Ptr{Cvoid}}),
                handle, task, Int64(max_batch), out))
    return out[]
end

value_count(plan) = ccall((:wnlqg_b200_plan_value_count, LIB), Int64, (Ptr{Cvoid},), plan)

"""Lane tensor sum_{k in [first,last)} value(k)/Nk on the Gamma-centred mesh (0-based indices)."""
function eval_mesh!(out::Vector{ComplexF64}, plan, mesh::NTuple{3, Int}, first::Integer, last::Integer)
    m = Int64[mesh...]
    check(ccall((:wnlqg_b200_eval_mesh, LIB), Cint, (Ptr{Cvoid}, Ptr{Int64}, Int64, Int64, Ptr{ComplexF64}),
                plan, m, Int64(first), Int64(last), out))
    return out
end

"""Batched ResponseNodeEvaluator: values of n fractional k-points, one column per point."""
function eval_points!(out::Matrix{ComplexF64}, plan, kpoints::Matrix{Float64})
    check(ccall((:wnlqg_b200_eval_points, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{ComplexF64}),
                plan, kpoints, Int64(size(kpoints, 2)), out))
    return out
end

"""wnlqg_autotune_report: the chosen eigensolver team and contraction tile, with the timings."""
struct AutotuneReport
    eigh_team::Int32
    energies_per_thread::Int32
    eigh_ms::NTuple{3, Float64}
    response_ms::NTuple{3, Float64}
    from_cache::Int32
    warm_start::Int32
    start_ms::NTuple{2, Float64}
    response_threads::Int32
    width_ms::NTuple{2, Float64}
    metric_shg_grid::Int32
    metric_shg_grid_ms::NTuple{3, Float64}
    shg_grid::Int32
    shg_grid_ms::NTuple{3, Float64}
    response_grid::Int32
    response_grid_ms::NTuple{3, Float64}
    eigh_grid::Int32
    eigh_grid_ms::NTuple{3, Float64}
end

"""Pick the eigensolver team and contraction tile by timing them on mesh indices [first, last)."""
function autotune!(plan, mesh::NTuple{3, Int}, first::Integer, last::Integer)
    m = Int64[mesh...]
    rep = Ref{AutotuneReport}()
    check(ccall((:wnlqg_b200_plan_autotune, LIB), Cint, (Ptr{Cvoid}, Ptr{Int64}, Int64, Int64, Ref{AutotuneReport}),
                plan, m, Int64(first), Int64(last), rep))
    return rep[]
end

"""Capture one weighted-points call on fixed device buffers (CuPtr addresses) as a CUDA graph;
refill the buffers and call graph_launch for each batch of adaptive nodes."""
function graph_capture_points(plan, kpoints_dev::Ptr{Float64}, weights_dev::Ptr{Float64}, n::Integer,
                              out_dev::Ptr{ComplexF64})
    g = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:wnlqg_b200_graph_capture_points_weighted, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{ComplexF64}, Ref{Ptr{Cvoid}}),
                plan, kpoints_dev, weights_dev, Int64(n), out_dev, g))
    return g[]
end

"""After synchronising the stream of an asynchronous call: pending device-side errors (a bounded
wait that gave up; a k-point failing the spectral isolation contract, thrown as ArgumentError)."""
plan_status(plan) = check(ccall((:wnlqg_b200_plan_status, LIB), Cint, (Ptr{Cvoid},), plan))

graph_launch(g, stream::Ptr{Cvoid} = C_NULL) =
    check(ccall((:wnlqg_b200_graph_launch, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), g, stream))
graph_destroy(g) = ccall((:wnlqg_b200_graph_destroy, LIB), Cint, (Ptr{Cvoid},), g)

plan_destroy(plan) = ccall((:wnlqg_b200_plan_destroy, LIB), Cint, (Ptr{Cvoid},), plan)
model_destroy(h) = ccall((:wnlqg_b200_model_destroy, LIB), Cint, (Ptr{Cvoid},), h)

end # module
