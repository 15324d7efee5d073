"""
    PeriDynB200

Julia binding of libperidyn_b200.so for PeriDyn (ABI version 2).  Load it
after PeriDyn; user scripts keep calling `run!`, `apply_solver!`,
`update_acc!`, `cal_damage`, ... unchanged.  Two ways in, selected through
PeriDyn's device switch `PeriDyn.DEVICE[]` (src/misc/const_macros.jl:10):

* `PeriDyn.DEVICE[] = :cuda` -- the reference's own CUDA dispatch point.
  `force_density!` (general_material.jl:240-256) calls
  `force_density_T!(f, y, limits, mat, Val{:cuda})` (general_material.jl:245,
  whose body throws at :388-390).  The method below, specialised on
  `CuMatrix{Float64}` arguments and therefore more specific than the
  reference's untyped one, runs the block's bond loop on the device
  arrays in place (`pd_force_density_device`), on CUDA.jl's current stream.

* `PeriDyn.DEVICE[] = :b200` -- the device-resident solver.  `run!` calls
  `apply_solver!(envs[id], solver)` every step (solvers.jl:148); the
  methods below (typed on `GeneralEnvironment`, so more specific than the
  reference's untyped `env`) advance the environment on the GPU
  (`pd_env_vv_steps`, `pd_env_qsdrag`) without copying the state back.  The
  host copy is brought up to date only where the host reads it:
  `printdata`, `print_data_file!` (and so `save_state!`), `cal_damage`,
  `update_acc!`, or an explicit `PeriDynB200.sync!(env)`.  A `Collect!`
  callback that reads the state should call `sync!` first, or set
  `PeriDynB200.SYNC_EVERY_STEP[] = true`.  `update_neighs!` rebuilds the
  contact neighbour lists on the device.  `set_device(:b200)` cannot be
  used for this (PeriDyn's `get_valid_device` maps every symbol other than
  `:cuda` to `:cpu`); assign `PeriDyn.DEVICE[]` directly or call
  `PeriDynB200.use_b200!()`.

Every `ccall` signature here mirrors include/peridyn_b200.h; the Python test
suite parses this file and checks each one (argument count and types, the
`MaterialDesc` field list, the constants) against the header, since no
Julia toolchain is available where the library is built.
"""
module PeriDynB200

using CUDA
using PeriDyn
import PeriDyn: force_density_T!, apply_solver!, update_acc!, cal_damage, printdata, print_data_file!,
                update_neighs!

const LIB = get(ENV, "PERIDYN_B200_LIB", joinpath(@__DIR__, "..", "peridyn_b200", "libperidyn_b200.so"))

const PD_ABI_VERSION = 2
const PD_MAT_BOND_BASED = Int32(0)
const PD_MAT_ORDINARY_STATE_BASED = Int32(1)
const PD_MAT_SKIP = Int32(2)
const PD_MAT_ELASTO_PLASTIC = Int32(3)
const PD_PREC_FP64_SERIAL = Int32(0)
const PD_PREC_FP64 = Int32(1)
const PD_PREC_FP32C = Int32(2)
const PD_BC_FIX = Int32(0)
const PD_BC_TOFRO = Int32(1)
const PD_CONTACT_12 = Int32(0)
const PD_CONTACT_11 = Int32(1)

"Mirror of `pd_material_desc` (include/peridyn_b200.h), field for field."
struct MaterialDesc
    kind::Int32
    ntypes::Int32
    type_start::Int64
    bond_stiffness::Ptr{Float64}
    bulk_modulus::Ptr{Float64}
    shear_modulus::Ptr{Float64}
    critical_stretch::Ptr{Float64}
    density::Ptr{Float64}
    horizon::Float64
    particle_size::Float64
    max_neigh::Int64
    plastic_psi::Ptr{Float64}
end

check(st) = st == 0 ? nothing :
    error("peridyn_b200: ", unsafe_string(ccall((:pd_last_error, LIB), Cstring, ())))

function __init__()
    v = ccall((:pd_abi_version, LIB), Cint, ())
    v == PD_ABI_VERSION || error("libperidyn_b200 has ABI version $v; this binding expects $PD_ABI_VERSION")
end

"Select the device-resident solver path (`PeriDyn.DEVICE[] = :b200`)."
use_b200!() = (PeriDyn.DEVICE[] = :b200; nothing)

"Precision (PD_PREC_*) and GPU of environments created from now on."
const PRECISION = Ref{Int32}(PD_PREC_FP64_SERIAL)
const GPU = Ref{Int32}(0)
"Copy the state back after every step (for `Collect!` callbacks that read it)."
const SYNC_EVERY_STEP = Ref(false)

"Device-resident mirror of one GeneralEnvironment."
mutable struct DeviceEnv
    h::Ptr{Cvoid}
    dirty::Bool   # the device state is newer than the host arrays
end

const ENVS = IdDict{Any,DeviceEnv}()
# single-block environments behind force_density_T!(..., Val{:cuda}), keyed
# by the block's GeneralMaterial
const BLOCKS = IdDict{Any,DeviceEnv}()

active(env) = PeriDyn.DEVICE[] === :b200 && env.state == 2

function material_kind(mat)
    mat isa PeriDyn.BondBasedMaterial && return PD_MAT_BOND_BASED
    mat isa PeriDyn.OrdinaryStateBasedMaterial && return PD_MAT_ORDINARY_STATE_BASED
    mat isa PeriDyn.ElastoPlasticSolidMaterial && return PD_MAT_ELASTO_PLASTIC
    mat isa PeriDyn.SkipMaterial && return PD_MAT_SKIP
    error("material $(typeof(mat)) has no B200 kernel")
end

"Append one material block (and its host-built family) to the device environment `h`."
function add_block!(h::Ptr{Cvoid}, mat)
    gen, spc = mat.general, mat.specific
    kind = material_kind(mat)
    nt = length(mat.type)
    z = zeros(nt, nt)
    c = kind == PD_MAT_BOND_BASED ? Matrix{Float64}(spc.bond_stiffness) : z
    K = kind in (PD_MAT_ORDINARY_STATE_BASED, PD_MAT_ELASTO_PLASTIC) ? Matrix{Float64}(spc.bulk_modulus) : z
    G = kind in (PD_MAT_ORDINARY_STATE_BASED, PD_MAT_ELASTO_PLASTIC) ? Matrix{Float64}(spc.shear_modulus) : z
    psi = kind == PD_MAT_ELASTO_PLASTIC ? Matrix{Float64}(spc.ψ) : z
    cs = kind == PD_MAT_SKIP ? z : Matrix{Float64}(spc.critical_stretch)
    rho = Vector{Float64}(Array(spc.density))
    x, y, v = Array{Float64}(gen.x), Array{Float64}(gen.y), Array{Float64}(gen.velocity)
    vol, typ = Vector{Float64}(Array(gen.volume)), Vector{Int64}(Array(gen.type))
    fam = Matrix{Int64}(Array(gen.family.x))
    intact = Matrix{UInt8}(Array(gen.intact.x))
    out = Ref{Int64}(0)
    GC.@preserve c K G psi cs rho begin
        d = MaterialDesc(kind, Int32(nt), first(mat.type), pointer(c), pointer(K), pointer(G), pointer(cs),
                         pointer(rho), gen.horizon, gen.particle_size, size(fam, 1), pointer(psi))
        check(ccall((:pd_env_add_block, LIB), Int32,
                    (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Int64},
                     Ref{MaterialDesc}, Ptr{Int64}),
                    h, size(x, 2), x, y, v, vol, typ, d, out))
    end
    # keep the family PeriDyn already built (reference layout: rows x n, 1-based, descending)
    check(ccall((:pd_env_set_family, LIB), Int32, (Ptr{Cvoid}, Int64, Int64, Ptr{Int64}, Ptr{UInt8}),
                h, out[], size(fam, 1), fam, intact))
    out[]
end

function create(dt; precision=PRECISION[], device=GPU[])
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:pd_env_create, LIB), Int32, (Ptr{Ptr{Cvoid}}, Int32, Int32, Float64),
                h, Int32(device), Int32(precision), Float64(dt)))
    h[]
end

"The device environment of `env`, built from its current host state on first use."
function device_env(env)
    get!(ENVS, env) do
        h = create(env.dt)
        for mat in env.material_blocks
            add_block!(h, mat)
        end
        for bc in env.boundary_conditions
            kind = bc isa PeriDyn.ToFroBC ? PD_BC_TOFRO : PD_BC_FIX
            bc isa Union{PeriDyn.FixBC,PeriDyn.ToFroBC} ||
                error("boundary condition $(typeof(bc)): use pd_env_add_scaled_bc / pd_env_add_container_bc")
            mask = Vector{UInt8}(Array(bc.bool))
            dims = Vector{UInt8}(Array(bc.dims))
            rate = kind == PD_BC_TOFRO ? Vector{Float64}(Array(bc.rate)) : zeros(3)
            freq = kind == PD_BC_TOFRO ? Float64(bc.freq) : Inf
            after = kind == PD_BC_TOFRO ? Int64(bc.applyafter) : Int64(0)
            check(ccall((:pd_env_add_bc, LIB), Int32,
                        (Ptr{Cvoid}, Int32, Ptr{UInt8}, Ptr{UInt8}, Ptr{Float64}, Float64, Int64, Int32, Ptr{Int64}),
                        h, kind, mask, dims, rate, freq, after, Int32(bc.onlyatstart), C_NULL))
        end
        for rm in env.short_range_contact
            if rm isa PeriDyn.ContactModel12
                b1 = findfirst(m -> m.type == rm.pair[1], env.material_blocks) - 1
                b2 = findfirst(m -> m.type == rm.pair[2], env.material_blocks) - 1
                kind, rows = PD_CONTACT_12, rm.max_neighs
            else
                b1 = findfirst(m -> m.general === rm.material, env.material_blocks) - 1
                b2, kind, rows = -1, PD_CONTACT_11, rm.max_neighs
            end
            check(ccall((:pd_env_add_contact, LIB), Int32,
                        (Ptr{Cvoid}, Int32, Int64, Int64, Float64, Float64, Float64, Float64, Int64, Ptr{Int64}),
                        h, kind, Int64(b1), Int64(b2), Float64(rm.exponent), Float64(rm.stifness),
                        Float64(rm.equi_dist), Float64(rm.distance), Int64(rows), C_NULL))
        end
        check(ccall((:pd_env_finalize, LIB), Int32, (Ptr{Cvoid},), h))
        # the host state as of now: y, v and the forces of the last update_acc!,
        # the BC snapshots of apply_bc_at0, the time step and the deformed gate
        y, v, f = Array{Float64}(env.y), Array{Float64}(env.v), Array{Float64}(env.f)
        check(ccall((:pd_env_set_state, LIB), Int32, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                    h, y, v, f))
        check(ccall((:pd_env_apply_bc_at0, LIB), Int32, (Ptr{Cvoid},), h))
        check(ccall((:pd_env_set_time_step, LIB), Int32, (Ptr{Cvoid}, Int64), h, Int64(env.time_step)))
        flags = UInt8[all(m.general.deformed) for m in env.material_blocks]
        check(ccall((:pd_env_set_deformed, LIB), Int32, (Ptr{Cvoid}, Ptr{UInt8}, Int32), h, flags, Int32(0)))
        DeviceEnv(h, false)
    end
end

"Bring the host arrays of `env` (y, v, f, p, time_step, intact flags, deformed) up to date."
function sync!(env)
    d = get(ENVS, env, nothing)
    (d === nothing || !d.dirty) && return env
    y, v, f, p = (Array{Float64}(undef, size(env.y)) for _ in 1:4)
    check(ccall((:pd_env_get_state, LIB), Int32, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                d.h, y, v, f, p))
    copyto!(env.y, y); copyto!(env.v, v); copyto!(env.f, f); copyto!(env.p, p)
    ts = Ref{Int64}(0)
    check(ccall((:pd_env_get_time_step, LIB), Int32, (Ptr{Cvoid}, Ptr{Int64}), d.h, ts))
    env.time_step = ts[]
    for (b, mat) in enumerate(env.material_blocks)
        fam = Array(mat.general.family.x)
        intact = Matrix{UInt8}(undef, size(fam))
        check(ccall((:pd_env_get_family, LIB), Int32, (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{UInt8}),
                    d.h, Int64(b - 1), fam, intact))
        copyto!(mat.general.intact.x, intact .!= 0)
    end
    flags = zeros(UInt8, length(env.material_blocks))
    check(ccall((:pd_env_deformed, LIB), Int32, (Ptr{Cvoid}, Ptr{UInt8}), d.h, flags))
    for (b, mat) in enumerate(env.material_blocks)
        flags[b] != 0 && (mat.general.deformed .= true)
    end
    d.dirty = false
    env
end

"Copy the host state (y, v, f) of `env` to the device, e.g. after the host changed it."
function push_state!(env)
    d = device_env(env)
    sync!(env)
    y, v, f = Array{Float64}(env.y), Array{Float64}(env.v), Array{Float64}(env.f)
    check(ccall((:pd_env_set_state, LIB), Int32, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                d.h, y, v, f))
    env
end

"Release the device copy of `env` (after a final `sync!`)."
function release!(env)
    d = pop!(ENVS, env, nothing)
    d === nothing || check(ccall((:pd_env_destroy, LIB), Int32, (Ptr{Cvoid},), d.h))
    nothing
end

# --- the device-resident solver (DEVICE[] === :b200) --------------------------

"apply_solver!(env, ::DSVelocityVerlet) (velocity_verlet.jl:27), reached from run! (solvers.jl:148)."
function apply_solver!(env::PeriDyn.GeneralEnvironment, solver::PeriDyn.DSVelocityVerlet)
    active(env) || return invoke(apply_solver!, Tuple{Any,PeriDyn.DSVelocityVerlet}, env, solver)
    d = device_env(env)
    check(ccall((:pd_env_vv_steps, LIB), Int32, (Ptr{Cvoid}, Int64), d.h, Int64(1)))
    env.time_step += 1
    d.dirty = true
    SYNC_EVERY_STEP[] && sync!(env)
    nothing
end

"apply_solver!(env, ::QSDrag) (minimize.jl:74): one minimize! on the device."
function apply_solver!(env::PeriDyn.GeneralEnvironment, s::PeriDyn.QSDrag)
    active(env) || return invoke(apply_solver!, Tuple{Any,PeriDyn.QSDrag}, env, s)
    d = device_env(env)
    it = Ref{Int64}(0)
    check(ccall((:pd_env_qsdrag, LIB), Int32, (Ptr{Cvoid}, Float64, Float64, Int64, Float64, Float64, Ptr{Int64}),
                d.h, Float64(s.step_size), Float64(s.drag), Int64(s.max_iter), Float64(s.x_tol), Float64(s.f_tol), it))
    d.dirty = true
    SYNC_EVERY_STEP[] && sync!(env)
    nothing
end

"update_acc!(env) (solvers.jl:320-336) on the device; the host receives f and p."
function update_acc!(env::PeriDyn.GeneralEnvironment)
    active(env) || return invoke(update_acc!, Tuple{Any}, env)
    d = device_env(env)
    check(ccall((:pd_env_update_acc, LIB), Int32, (Ptr{Cvoid},), d.h))
    d.dirty = true
    sync!(env)
    nothing
end

"update_neighs!(envs; max_part) (solvers.jl:351-361): contact neighbour lists rebuilt on the device."
function update_neighs!(envs::Vector{PeriDyn.GeneralEnvironment}; max_part=30)
    for env in envs
        if active(env)
            d = device_env(env)
            check(ccall((:pd_env_update_neighs, LIB), Int32, (Ptr{Cvoid}, Int64), d.h, Int64(max_part)))
        elseif env.state == 2
            invoke(update_neighs!, Tuple{Any}, [env]; max_part=max_part)
        end
    end
    nothing
end

"printdata(env) (environment.jl:308-320) after bringing the host copy up to date."
function printdata(env::PeriDyn.GeneralEnvironment)
    sync!(env)
    invoke(printdata, Tuple{Any}, env)
end

"print_data_file!(envs, prefix, i) (io.jl:107) after bringing the host copies up to date."
function print_data_file!(envs::Vector{PeriDyn.GeneralEnvironment}, file_prefix::String, i; ext::Symbol=:jld)
    foreach(sync!, envs)
    invoke(print_data_file!, Tuple{Array{PeriDyn.GeneralEnvironment},String,Any}, envs, file_prefix, i; ext=ext)
end

"cal_damage(env) (peri.jl:587-594) from the device's intact flags."
function cal_damage(env::PeriDyn.GeneralEnvironment)
    active(env) || return invoke(cal_damage, Tuple{Any}, env)
    d = device_env(env)
    out = zeros(Float64, size(env.y, 2))
    check(ccall((:pd_env_damage, LIB), Int32, (Ptr{Cvoid}, Ptr{Float64}), d.h, out))
    out
end

# --- the reference's CUDA dispatch point (DEVICE[] === :cuda) -----------------

"The single-block device environment standing for `mat` (families and flags stay on the device)."
function block_env(mat)
    get!(BLOCKS, mat.general) do
        h = create(1.0; precision=PD_PREC_FP64_SERIAL)
        add_block!(h, mat)
        check(ccall((:pd_env_finalize, LIB), Int32, (Ptr{Cvoid},), h))
        DeviceEnv(h, false)
    end
end

"""
force_density_T!(f, y, limits, mat, Val{:cuda}) (general_material.jl:245, :388-390) on the
CuArrays of the environment: the block's columns limits[1]:limits[2] of f receive its bond
forces, in place, on CUDA.jl's current stream; the block's intact flags live on the device
(`block_env`).
"""
function force_density_T!(f::CuMatrix{Float64}, y::CuMatrix{Float64}, limits, mat::PeriDyn.PeridynamicsMaterial,
                          ::Type{Val{:cuda}}; particles=nothing)
    particles === nothing || error("peridyn_b200: a particle subset is not supported")
    d = block_env(mat)
    off = 3 * (limits[1] - 1) + 1      # first element of the block's columns
    fp = reinterpret(CuPtr{Cvoid}, pointer(f, off))
    yp = reinterpret(CuPtr{Cvoid}, pointer(y, off))
    st = reinterpret(Ptr{Cvoid}, CUDA.stream().handle)
    check(ccall((:pd_force_density_device, LIB), Int32, (Ptr{Cvoid}, Int64, CuPtr{Cvoid}, CuPtr{Cvoid}, Ptr{Cvoid}),
                d.h, Int64(0), fp, yp, st))
    nothing
end

"The same for callers that may not allocate device memory during a step (`pd_force_density_device_static`)."
function force_density_static!(f::CuMatrix{Float64}, y::CuMatrix{Float64}, limits, mat::PeriDyn.PeridynamicsMaterial)
    d = block_env(mat)
    off = 3 * (limits[1] - 1) + 1
    fp = reinterpret(CuPtr{Cvoid}, pointer(f, off))
    yp = reinterpret(CuPtr{Cvoid}, pointer(y, off))
    st = reinterpret(Ptr{Cvoid}, CUDA.stream().handle)
    check(ccall((:pd_force_density_device_static, LIB), Int32,
                (Ptr{Cvoid}, Int64, CuPtr{Cvoid}, CuPtr{Cvoid}, Ptr{Cvoid}), d.h, Int64(0), fp, yp, st))
    nothing
end

"force_density_T!(f, y, limits, mat, Val{:b200}) on host arrays (force_density! with DEVICE[] === :b200)."
function force_density_T!(f, y, limits, mat::PeriDyn.PeridynamicsMaterial, ::Type{Val{:b200}}; particles=nothing)
    fd, yd = CuArray{Float64}(f), CuArray{Float64}(y)
    force_density_T!(fd, yd, limits, mat, Val{:cuda}; particles=particles)
    copyto!(f, Array(fd))
    nothing
end

end # module
