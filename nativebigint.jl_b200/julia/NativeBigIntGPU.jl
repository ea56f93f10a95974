# NativeBigIntGPU.jl — Julia binding of libnbgpu.so for NativeBigInt.jl.
#
# Drop-in for the fp-NTT branch of the reference's mpn multiply: the engine
# functions mul_fpntt2!/sqr_fpntt2! (src/fpntt.jl:982, :1016) keep their
# signatures and call the B200 engine through ccall.  Results are bit-identical
# to the CPU engine.  Karatsuba and basecase products stay on the CPU.
#
# Usage (inside NativeBigInt, after `include("fpntt.jl")`):
#     include("NativeBigIntGPU.jl"); using .NativeBigIntGPU
#     NativeBigIntGPU.install!()     # route mul_fpntt2!/sqr_fpntt2! to the GPU
module NativeBigIntGPU

const Limb = UInt64
const LIB = get(ENV, "NBGPU_LIB", joinpath(@__DIR__, "..", "lib", "libnbgpu.so"))

const NBG_ERANGE = Cint(2)

struct NBGError <: Exception
    code::Cint
    msg::String
end
Base.showerror(io::IO, e::NBGError) = print(io, "nbgpu error ", e.code, ": ", e.msg)

function check(rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:nbg_last_error, LIB), Cstring, ()))
    # the reference throws ArgumentError past 315*2^34 points (src/fpntt.jl:948-949)
    rc == NBG_ERANGE && throw(ArgumentError(msg))
    throw(NBGError(rc, msg))
end

# r[ro+1 .. ro+m+n] = a[ao+1 .. ao+m] * b[bo+1 .. bo+n]   (mul_fpntt2!, src/fpntt.jl:982)
function gpu_mul_fpntt2!(r::Memory{Limb}, ro::Int, a::Memory{Limb}, ao::Int, m::Int,
                         b::Memory{Limb}, bo::Int, n::Int)
    @boundscheck (ro + m + n <= length(r) && ao + m <= length(a) && bo + n <= length(b)) ||
        throw(BoundsError())
    GC.@preserve r a b begin
        rc = ccall((:nbg_mul, LIB), Cint,
                   (Ptr{Limb}, Ptr{Limb}, Int64, Ptr{Limb}, Int64),
                   pointer(r, ro + 1), pointer(a, ao + 1), m, pointer(b, bo + 1), n)
    end
    check(rc)
    return nothing
end

# r[ro+1 .. ro+2n] = a[ao+1 .. ao+n]^2   (sqr_fpntt2!, src/fpntt.jl:1016)
function gpu_sqr_fpntt2!(r::Memory{Limb}, ro::Int, a::Memory{Limb}, ao::Int, n::Int)
    @boundscheck (ro + 2n <= length(r) && ao + n <= length(a)) || throw(BoundsError())
    GC.@preserve r a begin
        rc = ccall((:nbg_sqr, LIB), Cint, (Ptr{Limb}, Ptr{Limb}, Int64),
                   pointer(r, ro + 1), pointer(a, ao + 1), n)
    end
    check(rc)
    return nothing
end

# r[ro+1 .. ro+k] = low k limbs of a*b (the full-product branch of mullo!,
# src/mul.jl:316-319) and of a^2 (sqrlo!, :361-364)
function gpu_mullo!(r::Memory{Limb}, ro::Int, a::Memory{Limb}, ao::Int, la::Int,
                    b::Memory{Limb}, bo::Int, lb::Int, k::Int)
    @boundscheck (ro + k <= length(r) && ao + la <= length(a) && bo + lb <= length(b)) || throw(BoundsError())
    GC.@preserve r a b begin
        rc = ccall((:nbg_mullo, LIB), Cint, (Ptr{Limb}, Ptr{Limb}, Int64, Ptr{Limb}, Int64, Int64),
                   pointer(r, ro + 1), pointer(a, ao + 1), la, pointer(b, bo + 1), lb, k)
    end
    check(rc)
    return nothing
end

function gpu_sqrlo!(r::Memory{Limb}, ro::Int, a::Memory{Limb}, ao::Int, la::Int, k::Int)
    @boundscheck (ro + k <= length(r) && ao + la <= length(a)) || throw(BoundsError())
    GC.@preserve r a begin
        rc = ccall((:nbg_sqrlo, LIB), Cint, (Ptr{Limb}, Ptr{Limb}, Int64, Int64),
                   pointer(r, ro + 1), pointer(a, ao + 1), la, k)
    end
    check(rc)
    return nothing
end

# Where an m x n product (m >= n) goes once the GPU is installed: the
# reference's CPU kernels below its NTT admission (src/mul.jl:12-26, :383-390)
# unless the product is large enough to pay for a GPU call.  The chunked
# Karatsuba path for n < MUL_FPNTT_MIN costs about m*n^0.585 limb operations
# there, so long unbalanced products with a small operand move to the GPU.
# Measured on B200 (bench.py --route): one host-buffer GPU call costs about
# 75 us and overtakes GMP's mpn_mul near m*n^0.585 = 1e5 (m = 1e4, n = 29:
# 101 us vs 133 us; m = 1e6, n = 63: 1.35 ms vs 19.6 ms).
const GPU_CHUNKED_MIN_WORK = 1.0e5   # m * n^0.585 above which a call pays off
route_to_gpu(m::Int, n::Int) = (n >= 64 && m + n >= 304) || m * Float64(n)^0.585 >= GPU_CHUNKED_MIN_WORK

# Batched products: descs as in include/nbgpu.h (nbg_desc); b == C_NULL squares a.
struct NbgDesc
    r::Ptr{Limb}
    a::Ptr{Limb}
    b::Ptr{Limb}
    m::Int64
    n::Int64
    bits_a::Int64
    bits_b::Int64
end

function gpu_mul_batch!(descs::Vector{NbgDesc})
    rc = ccall((:nbg_mul_batch, LIB), Cint, (Ptr{NbgDesc}, Int64), descs, length(descs))
    check(rc)
    return nothing
end

# Many powermod(b, e, m) calls with moduli of one size k (powermod_limbs on its
# Barrett branch, src/algorithms.jl:17-107): each chain's r gets b^e mod m
# (k limbs); b has at most k limbs, e is nonzero, m[k] != 0 and m > 1.
struct NbgPowmodDesc
    r::Ptr{Limb}
    b::Ptr{Limb}
    e::Ptr{Limb}
    m::Ptr{Limb}
    lb::Int64
    le::Int64
end

function gpu_powermod_batch!(rs::Vector{Memory{Limb}}, bs::Vector{Memory{Limb}}, es::Vector{Memory{Limb}},
                             ms::Vector{Memory{Limb}}, k::Int)
    n = length(ms)
    (length(rs) == n && length(bs) == n && length(es) == n) || throw(ArgumentError("one r, b, e per modulus"))
    GC.@preserve rs bs es ms begin
        descs = [NbgPowmodDesc(pointer(rs[i]), pointer(bs[i]), pointer(es[i]), pointer(ms[i]),
                               length(bs[i]), length(es[i])) for i in 1:n]
        rc = ccall((:nbg_powermod_batch, LIB), Cint, (Ptr{NbgPowmodDesc}, Int64, Int64), descs, n, k)
    end
    check(rc)
    return nothing
end

# Limbs of the value of little-endian base-bb chunks (radix_combine,
# src/nbig.jl:410-417): NBig parsing above its divide-and-conquer threshold.
function gpu_radix_combine(chunks::Vector{Limb}, bb::Limb)
    out = Memory{Limb}(undef, max(length(chunks), 1))
    len = Ref{Int64}(0)
    GC.@preserve out chunks begin
        rc = ccall((:nbg_radix_combine, LIB), Cint, (Ptr{Limb}, Int64, Ptr{Limb}, Int64, UInt64, Ref{Int64}),
                   pointer(out), length(out), pointer(chunks), length(chunks), bb, len)
    end
    check(rc)
    return out, Int(len[])
end

# radix_chunks_dc's power table (src/nbig.jl:394-399): [bb, bb^2, bb^4, ...]
# while the last entry is <= x, each square on the GPU (x as limbs, normalized).
function gpu_radix_powtab(bb::Limb, x::Vector{Limb})
    cap = 4 * length(x) + 64
    out = Memory{Limb}(undef, cap)
    maxe = 70
    offs = Vector{Int64}(undef, maxe + 1)
    ne = Ref{Int32}(0)
    GC.@preserve out offs x begin
        rc = ccall((:nbg_radix_powtab, LIB), Cint,
                   (Ptr{Limb}, Int64, Ptr{Int64}, Int32, UInt64, Ptr{Limb}, Int64, Ref{Int32}),
                   pointer(out), cap, pointer(offs), maxe, bb, pointer(x), length(x), ne)
    end
    check(rc)
    return [out[offs[i]+1:offs[i+1]] for i in 1:Int(ne[])]
end

# Per-call crossover of the drop-in hook: one host-buffer call (pageable
# Memory, copies included) against the reference's CPU engine.  Measured on
# B200 with bench.py --route (route_crossover: the GPU call against GMP on one
# host core times the reference's published mul!/mpn_mul ratio): a call costs
# 58 us at 152 limbs and 109 us at 4864; it overtakes the CPU engine near
# m + n = 5200 output limbs for balanced products, 3950 for m = 4n, and
# n = 3260 for squares.  Products at or above GPU_MIN_OUT_LIMBS output limbs
# (squares: GPU_MIN_SQR_LIMBS operand limbs) go to the GPU; smaller NTT-sized
# products keep the reference's CPU mul_fpntt2!/sqr_fpntt2!.
const GPU_MIN_OUT_LIMBS = Ref(4600)
const GPU_MIN_SQR_LIMBS = Ref(3300)
gpu_pays(m::Int, n::Int) = m + n >= GPU_MIN_OUT_LIMBS[]
gpu_pays_sqr(n::Int) = n >= GPU_MIN_SQR_LIMBS[]

# Replaces the engine entry points of the enclosing NativeBigInt module so that
# every NTT-sized mul!/sqr!/mul_bal! (src/mul.jl:134, :146, :161, :388-390) and
# NBig * (src/nbig.jl:124-140) at or above the crossover runs on the GPU.  The
# reference's own CPU methods stay reachable for the smaller products: they are
# called in the world age captured before the replacement
# (Base.invoke_in_world), so nothing of the CPU engine is copied.
# min_out_limbs / min_sqr_limbs override the measured crossover (0: every
# product on the GPU).
function install!(mod::Module = parentmodule(@__MODULE__); min_out_limbs::Int = GPU_MIN_OUT_LIMBS[],
                  min_sqr_limbs::Int = GPU_MIN_SQR_LIMBS[])
    GPU_MIN_OUT_LIMBS[] = min_out_limbs
    GPU_MIN_SQR_LIMBS[] = min_sqr_limbs
    world = Base.get_world_counter()
    cpu_mul = getfield(mod, :mul_fpntt2!)
    cpu_sqr = getfield(mod, :sqr_fpntt2!)
    @eval mod begin
        function mul_fpntt2!(r::Memory{Limb}, ro::Int, a::Memory{Limb}, ao::Int, m::Int, b::Memory{Limb}, bo::Int,
                             n::Int)
            if $(gpu_pays)(m, n)
                return $(gpu_mul_fpntt2!)(r, ro, a, ao, m, b, bo, n)
            end
            return Base.invoke_in_world($world, $cpu_mul, r, ro, a, ao, m, b, bo, n)
        end
        function sqr_fpntt2!(r::Memory{Limb}, ro::Int, a::Memory{Limb}, ao::Int, n::Int)
            if $(gpu_pays_sqr)(n)
                return $(gpu_sqr_fpntt2!)(r, ro, a, ao, n)
            end
            return Base.invoke_in_world($world, $cpu_sqr, r, ro, a, ao, n)
        end
    end
    return nothing
end

end # module
