"""
    PeriDynB200

Julia binding of libperidyn_b200.so for PeriDyn.  Loading it after PeriDyn
adds methods for the `Val{:cuda}` dispatch points and a device-resident
solver path; user scripts keep calling `run!`, `update_acc!`, etc.

This file is not exercised here (no Julia toolchain in the build image); the
same ABI is exercised from Python by the test suite.
"""
module PeriDynB200

using PeriDyn
import PeriDyn: force_density_T!, apply_solver!, update_acc!, cal_damage

const LIB = get(ENV, "PERIDYN_B200_LIB", joinpath(@__DIR__, "..", "peridyn_b200", "libperidyn_b200.so"))

const PD_MAT_BOND_BASED = Int32(0)
const PD_MAT_ORDINARY_STATE_BASED = Int32(1)
const PD_MAT_SKIP = Int32(2)
const PD_BC_FIX = Int32(0)
const PD_BC_TOFRO = Int32(1)
const PD_CONTACT_12 = Int32(0)
const PD_CONTACT_11 = Int32(1)

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
end

check(st) = st == 0 ? nothing :
    error("peridyn_b200: ", unsafe_string(ccall((:pd_last_error, LIB), Cstring, ())))

"Device-resident mirror of one GeneralEnvironment."
mutable struct DeviceEnv
    h::Ptr{Cvoid}
end

const ENVS = IdDict{Any,DeviceEnv}()

function material_kind(mat)
    mat isa PeriDyn.BondBasedMaterial && return PD_MAT_BOND_BASED
    mat isa PeriDyn.OrdinaryStateBasedMaterial && return PD_MAT_ORDINARY_STATE_BASED
    mat isa PeriDyn.SkipMaterial && return PD_MAT_SKIP
    error("material $(typeof(mat)) has no B200 kernel")
end

"Build the device environment for `env` (blocks, families, BCs, contacts)."
function device_env(env; precision::Integer=0, device::Integer=0)
    get!(ENVS, env) do
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:pd_env_create, LIB), Int32, (Ptr{Ptr{Cvoid}}, Int32, Int32, Float64),
                    h, device, precision, env.dt))
        for mat in env.material_blocks
            gen, spc = mat.general, mat.specific
            kind = material_kind(mat)
            nt = length(mat.type)
            z = zeros(nt, nt)
            c = kind == PD_MAT_BOND_BASED ? Matrix{Float64}(spc.bond_stiffness) : z
            K = kind == PD_MAT_ORDINARY_STATE_BASED ? Matrix{Float64}(spc.bulk_modulus) : z
            G = kind == PD_MAT_ORDINARY_STATE_BASED ? Matrix{Float64}(spc.shear_modulus) : z
            cs = Matrix{Float64}(spc.critical_stretch)
            rho = Vector{Float64}(spc.density)
            x, y, v = Array(gen.x), Array(gen.y), Array(gen.velocity)
            vol, typ = Array(gen.volume), Vector{Int64}(Array(gen.type))
            GC.@preserve c K G cs rho x y v vol typ begin
                d = MaterialDesc(kind, nt, first(mat.type), pointer(c), pointer(K), pointer(G), pointer(cs),
                                 pointer(rho), gen.horizon, gen.particle_size, size(gen.family.x, 1) + 1)
                out = Ref{Int64}(0)
                check(ccall((:pd_env_add_block, LIB), Int32,
                            (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                             Ptr{Int64}, Ref{MaterialDesc}, Ptr{Int64}),
                            h[], size(x, 2), x, y, v, vol, typ, d, out))
                # keep the family PeriDyn already built (reference layout)
                fam = Matrix{Int64}(gen.family.x)
                intact = Matrix{UInt8}(gen.intact.x)
                check(ccall((:pd_env_set_family, LIB), Int32,
                            (Ptr{Cvoid}, Int64, Int64, Ptr{Int64}, Ptr{UInt8}),
                            h[], out[], size(fam, 1), fam, intact))
            end
        end
        for bc in env.boundary_conditions
            kind = bc isa PeriDyn.FixBC ? PD_BC_FIX : PD_BC_TOFRO
            mask = Vector{UInt8}(Array(bc.bool))
            dims = Vector{UInt8}(Array(bc.dims))
            rate = kind == PD_BC_TOFRO ? Vector{Float64}(Array(bc.rate)) : zeros(3)
            freq = kind == PD_BC_TOFRO ? Float64(bc.freq) : Inf
            after = kind == PD_BC_TOFRO ? bc.applyafter : 0
            check(ccall((:pd_env_add_bc, LIB), Int32,
                        (Ptr{Cvoid}, Int32, Ptr{UInt8}, Ptr{UInt8}, Ptr{Float64}, Float64, Int64, Int32, Ptr{Int64}),
                        h[], kind, mask, dims, rate, freq, after, Int32(bc.onlyatstart), C_NULL))
        end
        blocks = IdDict(m.general => i - 1 for (i, m) in enumerate(env.material_blocks))
        for rm in env.short_range_contact
            if rm isa PeriDyn.ContactModel12
                b1 = findfirst(m -> m.type == rm.pair[1], env.material_blocks) - 1
                b2 = findfirst(m -> m.type == rm.pair[2], env.material_blocks) - 1
                kind, rows = PD_CONTACT_12, rm.max_neighs
            else
                b1, b2 = blocks[rm.material], -1
                kind, rows = PD_CONTACT_11, size(rm.neighs, 1)
            end
            check(ccall((:pd_env_add_contact, LIB), Int32,
                        (Ptr{Cvoid}, Int32, Int64, Int64, Float64, Float64, Float64, Float64, Int64, Ptr{Int64}),
                        h[], kind, b1, b2, rm.exponent, rm.stifness, rm.equi_dist, rm.distance, rows, C_NULL))
        end
        check(ccall((:pd_env_finalize, LIB), Int32, (Ptr{Cvoid},), h[]))
        DeviceEnv(h[])
    end
end

"Copy the host state (y, v, f) of `env` to the device."
push_state!(env, d::DeviceEnv) = check(ccall((:pd_env_set_state, LIB), Int32,
    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), d.h, Array(env.y), Array(env.v), Array(env.f)))

"Copy the device state back into `env` (y, v, f, p) and its time step."
function pull_state!(env, d::DeviceEnv)
    y, v, f, p = similar(Array(env.y)), similar(Array(env.v)), similar(Array(env.f)), similar(Array(env.p))
    check(ccall((:pd_env_get_state, LIB), Int32, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                                                 Ptr{Float64}), d.h, y, v, f, p))
    env.y .= y; env.v .= v; env.f .= f; env.p .= p
    ts = Ref{Int64}(0)
    check(ccall((:pd_env_get_time_step, LIB), Int32, (Ptr{Cvoid}, Ptr{Int64}), d.h, ts))
    env.time_step = ts[]
    nothing
end

# --- dispatch points --------------------------------------------------------

"apply_solver!(env, ::DSVelocityVerlet) on the device (velocity_verlet.jl:27)."
function apply_solver!(env, solver::PeriDyn.DSVelocityVerlet, ::Type{Val{:b200}})
    d = device_env(env)
    check(ccall((:pd_env_vv_steps, LIB), Int32, (Ptr{Cvoid}, Int64), d.h, 1))
    pull_state!(env, d)
end

"apply_solver!(env, ::QSDrag) on the device (minimize.jl:74)."
function apply_solver!(env, s::PeriDyn.QSDrag, ::Type{Val{:b200}})
    d = device_env(env)
    it = Ref{Int64}(0)
    check(ccall((:pd_env_qsdrag, LIB), Int32, (Ptr{Cvoid}, Float64, Float64, Int64, Float64, Float64, Ptr{Int64}),
                d.h, s.step_size, s.drag, s.max_iter, s.x_tol, s.f_tol, it))
    pull_state!(env, d)
end

"update_acc!(env) on the device (solvers.jl:320)."
function update_acc!(env, ::Type{Val{:b200}})
    d = device_env(env)
    push_state!(env, d)
    check(ccall((:pd_env_update_acc, LIB), Int32, (Ptr{Cvoid},), d.h))
    pull_state!(env, d)
end

"force_density_T!(f, y, limits, mat, Val{:cuda}) on CuArrays (general_material.jl:388)."
function force_density_T!(f, y, limits, mat::PeriDyn.PeridynamicsMaterial, ::Type{Val{:cuda}};
                          particles=nothing, env=nothing)
    env === nothing && error("pass env= so the block's device data can be found")
    d = device_env(env)
    block = findfirst(m -> m === mat, env.material_blocks) - 1
    check(ccall((:pd_force_density_device, LIB), Int32, (Ptr{Cvoid}, Int64, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}),
                d.h, block, pointer(f), pointer(y), C_NULL))
end

"cal_damage(env) from the device intact flags (peri.jl:587)."
function cal_damage(env, ::Type{Val{:b200}})
    d = device_env(env)
    out = zeros(size(env.y, 2))
    check(ccall((:pd_env_damage, LIB), Int32, (Ptr{Cvoid}, Ptr{Float64}), d.h, out))
    out
end

end # module
