// -*- C++ -*-
/// @file ir_emit.hpp
/// @brief Serialises a Loom kernel type (loom::vm::kernel_blank) into the
/// line-based text IR ("loomir") that the B200 code generator lowers to CUDA.
///
/// The walk reads only the compile-time facts that Loom's own front end
/// already computed (Loom src/vm/core.hpp):
///   * K::blocks            basic blocks after label optimisation and
///                          fall-through jumps (core.hpp:1012-1015, 805-829)
///   * K::labelmap          label -> block index, HALT = index_t(-1)
///                          (core.hpp:985, 991-993)
///   * K::reg_names/types   register file, Union for punned names
///                          (core.hpp:1003-1009, 257-283)
///   * K::input_vars/output_vars, K::index_t (core.hpp:947-950)
///   * parse_literal<Var>() literal values exactly as Loom parses them
///                          (core.hpp:443-467, common/string.hpp:311-372)
/// Every Compute op is mapped to an op name plus the functor's operand type;
/// the value semantics of each name are those of Loom src/vm/operators.hpp and
/// the std:: functors (standard_eval, core.hpp:740-750).
///
/// IR grammar (one item per line):
///   loomir 1
///   kernel <name>
///   index <type>
///   straight <0|1>
///   reg <idx> <name> <bytes> <type>[,<type>...]
///   input <reg> <type> <name>
///   output <reg> <type> <name>
///   block <idx> <label> <n_instr>
///   i <op> <optype> <dst> <arg>... [| <const>...]     Compute
///   j <target>                                         Jump
///   p <var> <target>...                                ParmJump
///   end
/// Operands: r<reg>:<type> (typed view of a register) or k<type>:<hexbits>
/// (literal).  Targets are block indices; -1 is HALT.
#pragma once

#include <vm/core.hpp>
#include <vm/operators.hpp>

#include "b200_ops.hpp"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <string_view>
#include <type_traits>

namespace loom::vm::b200::ir
{
// ---------------------------------------------------------------- types
template <typename T>
struct tname
{
    static_assert(sizeof(T) == 0, "type not supported by the B200 backend");
};

#define LOOM_B200_TNAME(T, S)                        \
    template <>                                      \
    struct tname<T>                                  \
    {                                                \
        static constexpr std::string_view value = S; \
    }
LOOM_B200_TNAME(bool, "b8");
LOOM_B200_TNAME(std::int8_t, "i8");
LOOM_B200_TNAME(std::uint8_t, "u8");
LOOM_B200_TNAME(std::int16_t, "i16");
LOOM_B200_TNAME(std::uint16_t, "u16");
LOOM_B200_TNAME(std::int32_t, "i32");
LOOM_B200_TNAME(std::uint32_t, "u32");
LOOM_B200_TNAME(long, "i64");
LOOM_B200_TNAME(unsigned long, "u64");
LOOM_B200_TNAME(long long, "i64");
LOOM_B200_TNAME(unsigned long long, "u64");
LOOM_B200_TNAME(float, "f32");
LOOM_B200_TNAME(double, "f64");
#undef LOOM_B200_TNAME

template <typename T>
inline constexpr std::string_view tname_v = tname<T>::value;

template <typename T>
struct reg_type_list
{
    static std::string
    str()
    {
        return std::string(tname_v<T>);
    }
};

template <typename... Ts>
struct reg_type_list<loom::Union<Ts...>>
{
    static std::string
    str()
    {
        std::string s;
        ((s += (s.empty() ? "" : ","), s += tname_v<Ts>), ...);
        return s;
    }
};

// ---------------------------------------------------------------- ops
/// Op descriptor: name, the functor's operand type list ("-" when the functor
/// is generic) and optional trailing constants.
template <typename Op>
struct op_info
{
    static_assert(sizeof(Op) == 0, "op not supported by the B200 backend");
};

#define LOOM_B200_STD_OP(FUNCTOR, NAME)                   \
    template <typename T>                                 \
    struct op_info<FUNCTOR<T>>                            \
    {                                                     \
        static constexpr std::string_view name = NAME;    \
        static std::string                                \
        optype()                                          \
        {                                                 \
            return std::string(tname_v<T>);               \
        }                                                 \
        static std::string                                \
        consts()                                          \
        {                                                 \
            return {};                                    \
        }                                                 \
    }
LOOM_B200_STD_OP(std::plus, "add");
LOOM_B200_STD_OP(std::minus, "sub");
LOOM_B200_STD_OP(std::multiplies, "mul");
LOOM_B200_STD_OP(std::divides, "div");
LOOM_B200_STD_OP(std::modulus, "mod");
LOOM_B200_STD_OP(std::negate, "neg");
LOOM_B200_STD_OP(std::equal_to, "eq");
LOOM_B200_STD_OP(std::not_equal_to, "ne");
LOOM_B200_STD_OP(std::greater, "gt");
LOOM_B200_STD_OP(std::less, "lt");
LOOM_B200_STD_OP(std::greater_equal, "ge");
LOOM_B200_STD_OP(std::less_equal, "le");
LOOM_B200_STD_OP(std::logical_and, "land");
LOOM_B200_STD_OP(std::logical_or, "lor");
LOOM_B200_STD_OP(std::logical_not, "lnot");
LOOM_B200_STD_OP(std::bit_and, "band");
LOOM_B200_STD_OP(std::bit_or, "bor");
LOOM_B200_STD_OP(std::bit_xor, "bxor");
LOOM_B200_STD_OP(std::bit_not, "bnot");
LOOM_B200_STD_OP(loom::vm::ops::lshift, "shl");
LOOM_B200_STD_OP(loom::vm::ops::rshift, "shr");
LOOM_B200_STD_OP(loom::vm::ops::abs, "abs");
LOOM_B200_STD_OP(loom::vm::ops::rsqrt, "rsqrt");
LOOM_B200_STD_OP(loom::vm::ops::max, "max");
LOOM_B200_STD_OP(loom::vm::ops::min, "min");
LOOM_B200_STD_OP(loom::vm::ops::round, "round");
LOOM_B200_STD_OP(loom::vm::ops::ceil, "ceil");
LOOM_B200_STD_OP(loom::vm::ops::floor, "floor");
LOOM_B200_STD_OP(loom::vm::ops::trunc, "trunc");
LOOM_B200_STD_OP(loom::vm::ops::sin, "sin");
LOOM_B200_STD_OP(loom::vm::ops::cos, "cos");
LOOM_B200_STD_OP(loom::vm::ops::sqrt, "sqrt");
LOOM_B200_STD_OP(loom::vm::ops::copysign, "copysign");
#undef LOOM_B200_STD_OP

#define LOOM_B200_GENERIC_OP(FUNCTOR, NAME)            \
    template <>                                        \
    struct op_info<FUNCTOR>                            \
    {                                                  \
        static constexpr std::string_view name = NAME; \
        static std::string                             \
        optype()                                       \
        {                                              \
            return "-";                                \
        }                                              \
        static std::string                             \
        consts()                                       \
        {                                              \
            return {};                                 \
        }                                              \
    }
LOOM_B200_GENERIC_OP(std::identity, "mov");
LOOM_B200_GENERIC_OP(loom::vm::ops::cmov, "cmov");
LOOM_B200_GENERIC_OP(loom::vm::ops::fma, "fma");
LOOM_B200_GENERIC_OP(loom::vm::ops::fms, "fms");
LOOM_B200_GENERIC_OP(loom::vm::ops::assert_fp, "assert_fp");
#undef LOOM_B200_GENERIC_OP

template <typename T>
std::string
literal_bits(const T v)
{
    std::uint64_t bits = 0;
    std::memcpy(&bits, &v, sizeof(T));
    std::ostringstream os;
    os << 'k' << tname_v<T> << ":0x" << std::hex << bits;
    return os.str();
}

/// ops::sct<T, I, L> selects a constant from a literal table
/// (Loom src/vm/operators.hpp:183-202).
template <typename T, std::integral I, typename L>
struct op_info<loom::vm::ops::sct<T, I, L>>
{
    static constexpr std::string_view name = "sct";
    static std::string
    optype()
    {
        return std::string(tname_v<T>) + "," + std::string(tname_v<I>);
    }
    static std::string
    consts()
    {
        std::string s;
        for(const T v: loom::vm::ops::sct<T, I, L>::values)
            s += " " + literal_bits<T>(v);
        return s;
    }
};

/// ops::slt<T, I> selects one of its register operands (operators.hpp:209-219).
template <typename T, std::integral I>
struct op_info<loom::vm::ops::slt<T, I>>
{
    static constexpr std::string_view name = "slt";
    static std::string
    optype()
    {
        return std::string(tname_v<T>) + "," + std::string(tname_v<I>);
    }
    static std::string
    consts()
    {
        return {};
    }
};

template <template <typename> typename F>
struct fname;
template <>
struct fname<std::logical_and>
{
    static constexpr std::string_view value = "land";
};
template <>
struct fname<std::logical_or>
{
    static constexpr std::string_view value = "lor";
};
template <>
struct fname<std::equal_to>
{
    static constexpr std::string_view value = "eq";
};
template <>
struct fname<std::not_equal_to>
{
    static constexpr std::string_view value = "ne";
};
template <>
struct fname<std::greater>
{
    static constexpr std::string_view value = "gt";
};
template <>
struct fname<std::less>
{
    static constexpr std::string_view value = "lt";
};
template <>
struct fname<std::greater_equal>
{
    static constexpr std::string_view value = "ge";
};
template <>
struct fname<std::less_equal>
{
    static constexpr std::string_view value = "le";
};

/// ops::pacc<T, I, Acc, Cmp>: p <- Acc(p, Cmp(x, y)) (operators.hpp:239-254).
template <typename T,
          std::integral I,
          template <typename> typename Acc,
          template <typename> typename Cmp>
struct op_info<loom::vm::ops::pacc<T, I, Acc, Cmp>>
{
    static constexpr std::string_view name = "pacc";
    static std::string
    optype()
    {
        return std::string(tname_v<T>) + "," + std::string(tname_v<I>) + "," +
               std::string(fname<Acc>::value) + "," +
               std::string(fname<Cmp>::value);
    }
    static std::string
    consts()
    {
        return {};
    }
};

/// Table lookup extension (b200_ops.hpp): dst <- word idx of the table as T.
template <typename T>
struct op_info<loom::vm::b200::ops::tab<T>>
{
    static constexpr std::string_view name = "tab";
    static std::string
    optype()
    {
        return std::string(tname_v<T>);
    }
    static std::string
    consts()
    {
        return {};
    }
};

// ---------------------------------------------------------------- walk
template <Kernel K>
struct emitter
{
    using reg_names = typename K::reg_names;
    using labelmap  = typename K::labelmap;
    using index_t   = typename K::index_t;

    template <typename Var>
    static std::string
    operand()
    {
        using T = vartype<Var>;
        if constexpr(is_literal_v<Var>)
            return literal_bits<T>(static_cast<T>(parse_literal<Var>().value()));
        else
        {
            constexpr std::size_t idx =
                typelist::index<varname<Var>, reg_names>;
            return "r" + std::to_string(idx) + ":" + std::string(tname_v<T>);
        }
    }

    static std::string
    target(const index_t t)
    {
        return t == K::halt_pos ? std::string("-1") : std::to_string(t);
    }

    template <typename I>
    struct instr;

    template <typename Op, typename Dst, typename... Args>
    struct instr<Compute<Op, Dst, Args...>>
    {
        static void
        emit(std::ostream& os)
        {
            using info = op_info<Op>;
            os << "i " << info::name << ' ' << info::optype() << ' ' << operand<Dst>();
            ((os << ' ' << operand<Args>()), ...);
            const std::string c = info::consts();
            if(!c.empty()) os << " |" << c;
            os << '\n';
        }
    };

    template <typename Target>
    struct instr<Jump<Target>>
    {
        static void
        emit(std::ostream& os)
        {
            os << "j " << target(typelist::lookup<Target, labelmap>::value)
               << '\n';
        }
    };

    template <typename Var, typename Labels>
    struct instr<ParmJump<Var, Labels>>
    {
        static void
        emit(std::ostream& os)
        {
            os << "p " << operand<Var>();
            targets(os, jmp_idxs<ParmJump<Var, Labels>, labelmap>{});
            os << '\n';
        }

        template <typename I, I... ts>
        static void
        targets(std::ostream& os, std::integer_sequence<I, ts...>)
        {
            ((os << ' ' << target(static_cast<index_t>(ts))), ...);
        }
    };

    template <typename... Is>
    static void
    emit_block(std::ostream& os,
               std::size_t   idx,
               std::string_view label,
               type_sequence<Is...>)
    {
        os << "block " << idx << ' ' << label << ' ' << sizeof...(Is) << '\n';
        (instr<Is>::emit(os), ...);
    }

    template <typename... Blocks>
    static void
    emit_blocks(std::ostream& os, type_sequence<Blocks...>)
    {
        std::size_t idx = 0;
        // labels: START for block 0, then stated labels in order
        std::string names[sizeof...(Blocks)];
        label_names(names, typename K::labels{});
        ((emit_block(os, idx, names[idx], Blocks{}), ++idx), ...);
    }

    template <std::size_t N, typename... Ls>
    static void
    label_names(std::string (&names)[N], type_sequence<Ls...>)
    {
        std::size_t i = 0;
        ((i < N ? (names[i] = std::string(cs2sv<typename Ls::name>), 0) : 0,
          ++i),
         ...);
        for(; i < N; ++i) names[i] = "B" + std::to_string(i);
    }

    template <typename... Ns, typename... Ts>
    static void
    emit_regs(std::ostream& os, type_sequence<Ns...>, type_sequence<Ts...>)
    {
        std::size_t idx = 0;
        ((os << "reg " << idx++ << ' ' << cs2sv<Ns> << ' '
             << register_size<Ts>::value << ' ' << reg_type_list<Ts>::str()
             << '\n'),
         ...);
    }

    template <typename... Vs>
    static void
    emit_vars(std::ostream& os, std::string_view kind, type_sequence<Vs...>)
    {
        ((os << kind << ' ' << typelist::index<varname<Vs>, reg_names> << ' '
             << tname_v<vartype<Vs>> << ' ' << varview<Vs> << '\n'),
         ...);
    }

    static std::string
    emit(std::string_view name)
    {
        std::ostringstream os;
        os << "loomir 1\n";
        os << "kernel " << name << '\n';
        os << "index " << tname_v<index_t> << '\n';
        os << "straight " << (K::is_straightline ? 1 : 0) << '\n';
        emit_regs(os, reg_names{}, typename K::reg_types{});
        emit_vars(os, "input", typename K::input_vars{});
        emit_vars(os, "output", typename K::output_vars{});
        emit_blocks(os, typename K::blocks{});
        os << "end\n";
        return os.str();
    }
};

/// @brief Text IR of kernel @p K under the registry name @p name.
template <Kernel K>
std::string
emit(std::string_view name)
{
    return emitter<K>::emit(name);
}

/// @brief FNV-1a (64-bit) of the IR text without its `kernel` line, as 16
/// hex digits: identifies the program independently of its registry name.
inline std::string
structural_digest(std::string_view text)
{
    std::uint64_t h = 0xcbf29ce484222325ull;
    std::size_t   pos = 0;
    while(pos < text.size())
    {
        std::size_t end = text.find('\n', pos);
        end             = end == std::string_view::npos ? text.size() : end + 1;
        const std::string_view ln = text.substr(pos, end - pos);
        if(ln.substr(0, 7) != "kernel ")
            for(const unsigned char c: ln)
            {
                h ^= c;
                h *= 0x100000001b3ull;
            }
        pos = end;
    }
    char buf[17];
    std::snprintf(buf, sizeof buf, "%016llx", static_cast<unsigned long long>(h));
    return buf;
}

/// @brief Structural digest of kernel @p K.
template <Kernel K>
std::string
digest()
{
    return structural_digest(emit<K>(""));
}
} // namespace loom::vm::b200::ir
