"""
    ElemCoGPU

Julia side of libecgpu: `ccall` bindings of include/ecgpu.h and drop-in
replacements for ElemCo.jl's closed-shell `calc_cc`, `calc_pertT` and
`calc_lm_cc` (src/cc/cc.jl:2451, src/cc/cc_triples.jl:11,
src/cc/cc_lagrange.jl:1120).  They read the same inputs (the `mmL` DF factors
or EC.fd, the Fock matrix) and write the same scratch files (`T_vo`,
`T_vvoo`, `U_vo`, `U_vvoo`, `cc_amplitudes_*`, `cc_multipliers_*`), so the
rest of `ccdriver` is unchanged.  `eval_cc_groundstate`
(src/cc/ccdriver.jl:348-393) calls them in place of `calc_cc`, `calc_lm_cc`
and `calc_pertT` when a GPU context is set.

Host arrays are passed as `Ptr{Cdouble}` inside `GC.@preserve`; Julia's
column-major layout is the library's layout.  Status codes other than 0 raise
`ErrorException(ecg_last_error)`.
"""
module ElemCoGPU

export GPUContext, gpu_calc_cc, gpu_calc_pertT, gpu_calc_lm_cc, set_option!, tune_load!, tune_save,
       ShellArrays, int1e, int2c2e, int3c2e, DFFactors, df_fock, df_mo, release!

const libecgpu = get(ENV, "ECGPU_LIB", joinpath(@__DIR__, "..", "ecgpu", "libecgpu.so"))

struct CcOpts
  thr::Cdouble
  conven::Cdouble
  maxit::Int32
  shifts::Cdouble
  shiftp::Cdouble
  maxdiis::Int32
  resthr::Cdouble
  diis_dot::Int32   # ECG_DIIS_CS = 0 (the reference's closed-shell dots), ECG_DIIS_PLAIN = 1
end

const ECG_DIIS_CS = Int32(0)
const ECG_DIIS_PLAIN = Int32(1)
const ECG_OPT_TRIPLES_BATCH = Int32(1)
const ECG_OPT_TC_WAIT_NS = Int32(2)
const ECG_OPT_AUTOTUNE = Int32(3)
const ECG_INT_OVERLAP = Int32(0)
const ECG_INT_KINETIC = Int32(1)
const ECG_INT_NUCLEAR = Int32(2)
const ECG_INT_DIPOLE = Int32(3)

"""
    GPUContext(device=0)

One device-resident closed-shell CC problem (`ecg_ctx`); freed by a finalizer.
"""
mutable struct GPUContext
  ptr::Ptr{Cvoid}
  no::Int
  nv::Int
  nq::Int
  function GPUContext(device::Integer=0)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    st = ccall((:ecg_create, libecgpu), Cint, (Cint, Ptr{Ptr{Cvoid}}), device, r)
    st == 0 || error(unsafe_string(ccall((:ecg_last_error, libecgpu), Cstring, (Ptr{Cvoid},), C_NULL)))
    ctx = new(r[], 0, 0, 0)
    finalizer(c -> (c.ptr != C_NULL && ccall((:ecg_destroy, libecgpu), Cint, (Ptr{Cvoid},), c.ptr); c.ptr = C_NULL), ctx)
    return ctx
  end
end

function check(ctx::GPUContext, st::Cint)
  st == 0 && return nothing
  error("libecgpu status $st: " * unsafe_string(ccall((:ecg_last_error, libecgpu), Cstring, (Ptr{Cvoid},), ctx.ptr)))
end

function options(EC)
  cc = EC.options.cc
  d = EC.options.diis
  return CcOpts(cc.thr, cc.conven, Int32(cc.maxit), cc.shifts, cc.shiftp, Int32(d.maxdiis), d.resthr,
                ECG_DIIS_CS)
end

"""
    set_option!(ctx, key, value)

`ecg_set_option`: `ECG_OPT_TRIPLES_BATCH` (triplets per (T) batch),
`ECG_OPT_TC_WAIT_NS` (tensor-core GEMM wait bound), `ECG_OPT_AUTOTUNE`.
"""
set_option!(ctx::GPUContext, key::Integer, value::Integer) =
  check(ctx, ccall((:ecg_set_option, libecgpu), Cint, (Ptr{Cvoid}, Int32, Int64),
                   ctx.ptr, key, value))

"""
    tune_load!(ctx, path) / tune_save(ctx, path)

Merge a GEMM tuning table ("key value" lines, e.g. ecgpu/tuning/b200.txt)
into the process-wide table, or write the table; return its size.
"""
function tune_load!(ctx::GPUContext, path::AbstractString)
  n = Ref{Int64}(0)
  check(ctx, ccall((:ecg_tune_load, libecgpu), Cint, (Ptr{Cvoid}, Cstring, Ref{Int64}), ctx.ptr, path, n))
  return n[]
end
function tune_save(ctx::GPUContext, path::AbstractString)
  n = Ref{Int64}(0)
  check(ctx, ccall((:ecg_tune_save, libecgpu), Cint, (Ptr{Cvoid}, Cstring, Ref{Int64}), ctx.ptr, path, n))
  return n[]
end

# Shells of an ElemCo.jl BasisSet in the plain arrays of `ecg_shells`
# (per shell: l, primitive count, centre; exponents and coefficients of the
# basis file, shell after shell).  `shells` yields (l, centre, exps, coefs).
struct ShellArrays
  l::Vector{Int32}
  nprim::Vector{Int32}
  centre::Vector{Cdouble}
  exps::Vector{Cdouble}
  coefs::Vector{Cdouble}
end
function ShellArrays(shells)
  l = Int32[]; np = Int32[]; cen = Cdouble[]; ex = Cdouble[]; co = Cdouble[]
  for (ls, c, e, k) in shells
    push!(l, ls); push!(np, length(e)); append!(cen, c); append!(ex, e); append!(co, k)
  end
  return ShellArrays(l, np, cen, ex, co)
end
struct CShells
  nshell::Int32
  l::Ptr{Int32}
  nprim::Ptr{Int32}
  centre::Ptr{Cdouble}
  exps::Ptr{Cdouble}
  coefs::Ptr{Cdouble}
end
cshells(s::ShellArrays) = CShells(length(s.l), pointer(s.l), pointer(s.nprim), pointer(s.centre),
                                  pointer(s.exps), pointer(s.coefs))
function nbf(s::ShellArrays)
  n = Ref{Int32}(0)
  GC.@preserve s ccall((:ecg_shells_nbf, libecgpu), Cint, (Ref{CShells}, Ref{Int32}), cshells(s), n)
  return Int(n[])
end

"""
    int1e(ctx, kind, basis; charges, xyz, origin) -> Matrix (or 3 matrices for dipoles)

Overlap, kinetic, nuclear attraction or dipole integrals over real solid
harmonics (`ecg_int1e`; libcint int1e_ovlp/kin/nuc in src/system/integrals_2idx.jl).
"""
function int1e(ctx::GPUContext, kind::Integer, b::ShellArrays;
               charges=Cdouble[], xyz=Cdouble[], origin=Cdouble[0, 0, 0])
  n = nbf(b)
  out = zeros(n, n, kind == ECG_INT_DIPOLE ? 3 : 1)
  q = Vector{Cdouble}(charges); r = Vector{Cdouble}(vec(xyz)); o = Vector{Cdouble}(origin)
  GC.@preserve b q r o out check(ctx, ccall((:ecg_int1e, libecgpu), Cint,
      (Ptr{Cvoid}, Int32, Ref{CShells}, Int32, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
      ctx.ptr, kind, cshells(b), length(q), q, r, o, out))
  return kind == ECG_INT_DIPOLE ? out : out[:, :, 1]
end

"""
    int2c2e(ctx, fit) / int3c2e(ctx, ao, fit)

The fitting metric (P|Q) and the three-index integrals (mn|P) as `[m,n,P]`
(`ecg_int2c2e`, `ecg_int3c2e`; eri_2e2idx / eri_2e3idx of the reference).
"""
function int2c2e(ctx::GPUContext, f::ShellArrays)
  n = nbf(f)
  out = zeros(n, n)
  GC.@preserve f out check(ctx, ccall((:ecg_int2c2e, libecgpu), Cint,
      (Ptr{Cvoid}, Ref{CShells}, Ptr{Cdouble}), ctx.ptr, cshells(f), out))
  return out
end
function int3c2e(ctx::GPUContext, a::ShellArrays, f::ShellArrays)
  out = zeros(nbf(a), nbf(a), nbf(f))
  GC.@preserve a f out check(ctx, ccall((:ecg_int3c2e, libecgpu), Cint,
      (Ptr{Cvoid}, Ref{CShells}, Ref{CShells}, Ptr{Cdouble}), ctx.ptr, cshells(a), cshells(f), out))
  return out
end

"""
    DFFactors(ctx, ao, fit, M)

Density-fitted factors `AAL[m,n,L] = sum_P (mn|P) M[P,L]` kept on the device
(`ecg_df_create`; generate_AO_DF_integrals, src/integrals/dftools.jl:28-84),
`M` with `M M' = (P|Q)^-1` (the pivoted Cholesky of `int2c2e`).  Release with
`release!` before the context.
"""
mutable struct DFFactors
  ptr::Ptr{Cvoid}
  ctx::GPUContext
  nao::Int
  nL::Int
end
function DFFactors(ctx::GPUContext, a::ShellArrays, f::ShellArrays, M::Matrix{Float64})
  @assert size(M, 1) == nbf(f)
  h = Ref{Ptr{Cvoid}}(C_NULL)
  GC.@preserve a f M check(ctx, ccall((:ecg_df_create, libecgpu), Cint,
      (Ptr{Cvoid}, Ref{CShells}, Ref{CShells}, Ptr{Cdouble}, Int64, Ref{Ptr{Cvoid}}),
      ctx.ptr, cshells(a), cshells(f), M, size(M, 2), h))
  return DFFactors(h[], ctx, nbf(a), size(M, 2))
end

"""
    df_fock(df, h, Cocc)

Closed-shell Fock matrix `h + 2J - K` from the occupied orbitals (`ecg_df_fock`;
gen_dffock, src/scf/fockfactory.jl:202-245).
"""
function df_fock(df::DFFactors, h::Matrix{Float64}, Cocc::Matrix{Float64})
  F = zeros(df.nao, df.nao)
  GC.@preserve h Cocc F check(df.ctx, ccall((:ecg_df_fock, libecgpu), Cint,
      (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Int64, Ptr{Cdouble}),
      df.ptr, h, Cocc, size(Cocc, 2), F))
  return F
end

"""
    df_mo(df, C)

MO three-index factors `B[p,q,L]` (`ecg_df_mo`; generate_3idx_integrals,
src/integrals/dftools.jl:92-136, the `mmL` file).
"""
function df_mo(df::DFFactors, C::Matrix{Float64})
  nmo = size(C, 2)
  B = zeros(nmo, nmo, df.nL)
  GC.@preserve C B check(df.ctx, ccall((:ecg_df_mo, libecgpu), Cint,
      (Ptr{Cvoid}, Ptr{Cdouble}, Int64, Ptr{Cdouble}), df.ptr, C, nmo, B))
  return B
end

function release!(df::DFFactors)
  if df.ptr != C_NULL
    ccall((:ecg_df_destroy, libecgpu), Cint, (Ptr{Cvoid},), df.ptr)
    df.ptr = C_NULL
  end
  return nothing
end

"""
    set_system!(ctx, B, h1, e0, nocc)

Upload `B[p,q,L]` (the `mmL` file, src/integrals/dftools.jl:92-134), the
one-electron integrals and the core energy (`ecg_set_system`).
"""
function set_system!(ctx::GPUContext, B::Array{Float64,3}, h1::Matrix{Float64}, e0::Float64, nocc::Integer)
  n = size(B, 1)
  @assert size(B, 2) == n && size(h1) == (n, n)
  ctx.no, ctx.nv, ctx.nq = nocc, n - nocc, size(B, 3)
  GC.@preserve B h1 check(ctx, ccall((:ecg_set_system, libecgpu), Cint,
      (Ptr{Cvoid}, Int32, Int32, Int32, Ptr{Cdouble}, Ptr{Cdouble}, Cdouble),
      ctx.ptr, ctx.no, ctx.nv, ctx.nq, B, h1, e0))
  return ctx
end

function mp2!(ctx::GPUContext)
  T1 = zeros(ctx.nv, ctx.no)
  T2 = zeros(ctx.nv, ctx.nv, ctx.no, ctx.no)
  e = Ref{Cdouble}(0.0)
  GC.@preserve T1 T2 check(ctx, ccall((:ecg_mp2, libecgpu), Cint,
      (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{Cdouble}), ctx.ptr, T1, T2, e))
  return e[], T1, T2
end

function cc_solve!(ctx::GPUContext, T1, T2, dc::Bool, o::CcOpts)
  out = zeros(5)
  it = Ref{Int32}(0)
  conv = Ref{Int32}(0)
  GC.@preserve T1 T2 out check(ctx, ccall((:ecg_cc_solve, libecgpu), Cint,
      (Ptr{Cvoid}, Cint, Ref{CcOpts}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{Int32}, Ref{Int32}),
      ctx.ptr, dc, o, T1, T2, out, it, conv))
  return out, Int(it[]), conv[] != 0
end

function pert_t(ctx::GPUContext, T1, T2)
  e = Ref{Cdouble}(0.0); eb = Ref{Cdouble}(0.0)
  GC.@preserve T1 T2 check(ctx, ccall((:ecg_pert_t, libecgpu), Cint,
      (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{Cdouble}, Ref{Cdouble}), ctx.ptr, T1, T2, e, eb))
  return e[], eb[]
end

function lambda_pert_t(ctx::GPUContext, T1, T2, U1, U2)
  e = Ref{Cdouble}(0.0); eb = Ref{Cdouble}(0.0)
  GC.@preserve T1 T2 U1 U2 check(ctx, ccall((:ecg_lambda_pert_t, libecgpu), Cint,
      (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ref{Cdouble}, Ref{Cdouble}),
      ctx.ptr, T1, T2, U1, U2, e, eb))
  return e[], eb[]
end

function lambda_solve!(ctx::GPUContext, T1, T2, dc::Bool, o::CcOpts)
  U1 = zeros(ctx.nv, ctx.no)
  U2 = zeros(ctx.nv, ctx.nv, ctx.no, ctx.no)
  out = zeros(3)
  it = Ref{Int32}(0); conv = Ref{Int32}(0)
  GC.@preserve T1 T2 U1 U2 out check(ctx, ccall((:ecg_lambda_solve, libecgpu), Cint,
      (Ptr{Cvoid}, Cint, Ref{CcOpts}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
       Ptr{Cdouble}, Ref{Int32}, Ref{Int32}),
      ctx.ptr, dc, o, T1, T2, U1, U2, out, it, conv))
  return U1, U2, Int(it[]), conv[] != 0
end

# ---------------------------------------------------------------- drop-ins
# These use ElemCo's own helpers (passed in as the module `EM`, i.e.
# `ElemCo`), so this file loads without ElemCo installed.

"""
    df_factors(EM, EC)

`mmL` DF factors for EC.fd: the file written by @dfints/dfdump, or — for an
FCIDUMP — the Cholesky decomposition of src/integrals/decomptools.jl:22-52.
"""
function df_factors(EM, EC)
  if !EM.ECInfos.file_exists(EC, "mmL")
    EM.DecompTools.calc_integrals_decomposition(EC)
  end
  return EM.TensorTools.load3idx(EC, "mmL")
end

function context(EM, EC)
  ctx = get!(EC.options.gpu, :ctx) do
    c = GPUContext(get(EC.options.gpu, :device, 0))
    table = joinpath(@__DIR__, "..", "ecgpu", "tuning", "b200.txt")
    isfile(table) && tune_load!(c, table)   # the packaged B200 GEMM tuning table
    c
  end
  SP = EC.space
  set_system!(ctx, df_factors(EM, EC), EM.FciDumps.integ1(EC.fd), EC.fd.int0, length(SP['o']))
  return ctx
end

"""
    gpu_calc_cc(EM, EC, method) -> OutDict

Closed-shell `calc_cc` (src/cc/cc.jl:2451-2516) on the GPU: starts from the
`T_vo`/`T_vvoo` MP2 guess, writes the converged amplitudes back to the same
files and returns the Hylleraas energies.
"""
function gpu_calc_cc(EM, EC, method)
  ctx = context(EM, EC)
  dc = method.theory[1:2] == "DC"
  T1 = EM.TensorTools.load2idx(EC, "T_vo")
  T2 = EM.TensorTools.load4idx(EC, "T_vvoo")
  out, it, conv = cc_solve!(ctx, T1, T2, dc, options(EC))
  conv || println("WARNING: CC iterations did not converge!")
  EM.TensorTools.save!(EC, "T_vo", T1)
  EM.TensorTools.save!(EC, "T_vvoo", T2)
  EM.CCTools.try2save_singles!(EC, T1)
  EM.CCTools.try2save_doubles!(EC, T2)
  return EM.OutDict("E"=>out[1], "ESS"=>out[2], "EOS"=>out[3], "EO"=>0.0)
end

"""
    gpu_calc_lm_cc(EM, EC, method)

Closed-shell `calc_lm_cc` (src/cc/cc_lagrange.jl:1120-1153): writes `U_vo`,
`U_vvoo` and the `cc_multipliers_*` files.
"""
function gpu_calc_lm_cc(EM, EC, method)
  ctx = context(EM, EC)
  dc = (method.theory == "DC" || last(method.theory, 2) == "DC")
  T1 = EM.TensorTools.load2idx(EC, "T_vo")
  T2 = EM.TensorTools.load4idx(EC, "T_vvoo")
  U1, U2, it, conv = lambda_solve!(ctx, T1, T2, dc, options(EC))
  conv || println("WARNING: CC-LM iterations did not converge!")
  EM.TensorTools.save!(EC, "U_vo", U1)
  EM.TensorTools.save!(EC, "U_vvoo", U2)
  EM.CCTools.try2save_singles!(EC, U1; type="LM")
  EM.CCTools.try2save_doubles!(EC, U2; type="LM")
  return nothing
end

"""
    gpu_calc_pertT(EM, EC, method) -> OutDict("ET3"=>..., "ET3b"=>...)

Closed-shell (T) / Λ(T) (src/cc/cc_triples.jl:11-30, :39-295).
"""
function gpu_calc_pertT(EM, EC, method)
  ctx = context(EM, EC)
  T1 = EM.TensorTools.load2idx(EC, "T_vo")
  T2 = EM.TensorTools.load4idx(EC, "T_vvoo")
  if EM.ECMethods.has_prefix(method, "Λ")
    U1 = EM.TensorTools.load2idx(EC, "U_vo")
    U2 = EM.TensorTools.load4idx(EC, "U_vvoo")
    e, eb = lambda_pert_t(ctx, T1, T2, U1, U2)
  else
    e, eb = pert_t(ctx, T1, T2)
  end
  return EM.OutDict("ET3"=>e, "ET3b"=>eb)
end

end # module
