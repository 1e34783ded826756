// Generated by loom_b200.codegen: the kernels compiled into libloom_b200.

#include "../runtime_iface.h"

extern const loom_b200::KernelEntry loom_b200_entry_abs_f32;
extern const loom_b200::KernelEntry loom_b200_entry_arithmetic_f32;
extern const loom_b200::KernelEntry loom_b200_entry_arithmetic_f64;
extern const loom_b200::KernelEntry loom_b200_entry_bit_and_u32;
extern const loom_b200::KernelEntry loom_b200_entry_bit_not_u32;
extern const loom_b200::KernelEntry loom_b200_entry_bit_not_u8;
extern const loom_b200::KernelEntry loom_b200_entry_bit_or_u64;
extern const loom_b200::KernelEntry loom_b200_entry_bit_xor_u16;
extern const loom_b200::KernelEntry loom_b200_entry_bool_and_u32;
extern const loom_b200::KernelEntry loom_b200_entry_bool_not_u8;
extern const loom_b200::KernelEntry loom_b200_entry_bool_or_u64;
extern const loom_b200::KernelEntry loom_b200_entry_bump_u32;
extern const loom_b200::KernelEntry loom_b200_entry_canonical_f32;
extern const loom_b200::KernelEntry loom_b200_entry_ceilfloor_f32;
extern const loom_b200::KernelEntry loom_b200_entry_collatz_u64;
extern const loom_b200::KernelEntry loom_b200_entry_cross_f32;
extern const loom_b200::KernelEntry loom_b200_entry_fac_u32;
extern const loom_b200::KernelEntry loom_b200_entry_fac_u64;
extern const loom_b200::KernelEntry loom_b200_entry_fib_u32;
extern const loom_b200::KernelEntry loom_b200_entry_fib_u64;
extern const loom_b200::KernelEntry loom_b200_entry_increment_i16;
extern const loom_b200::KernelEntry loom_b200_entry_increment_i32;
extern const loom_b200::KernelEntry loom_b200_entry_increment_u64;
extern const loom_b200::KernelEntry loom_b200_entry_increment_u8;
extern const loom_b200::KernelEntry loom_b200_entry_jmp4_f32;
extern const loom_b200::KernelEntry loom_b200_entry_jmp4_u16;
extern const loom_b200::KernelEntry loom_b200_entry_jmp4_u64;
extern const loom_b200::KernelEntry loom_b200_entry_lshift_u16;
extern const loom_b200::KernelEntry loom_b200_entry_lshift_u32;
extern const loom_b200::KernelEntry loom_b200_entry_lshift_u64;
extern const loom_b200::KernelEntry loom_b200_entry_minmax_f32;
extern const loom_b200::KernelEntry loom_b200_entry_minmax_f64;
extern const loom_b200::KernelEntry loom_b200_entry_norm_f32;
extern const loom_b200::KernelEntry loom_b200_entry_primary_const_256;
extern const loom_b200::KernelEntry loom_b200_entry_primary_const_b20_256;
extern const loom_b200::KernelEntry loom_b200_entry_pt2_const_40;
extern const loom_b200::KernelEntry loom_b200_entry_pt2_const_512;
extern const loom_b200::KernelEntry loom_b200_entry_pt_const_40;
extern const loom_b200::KernelEntry loom_b200_entry_pt_const_512;
extern const loom_b200::KernelEntry loom_b200_entry_rotl32_u32;
extern const loom_b200::KernelEntry loom_b200_entry_rshift_u16;
extern const loom_b200::KernelEntry loom_b200_entry_rshift_u32;
extern const loom_b200::KernelEntry loom_b200_entry_rshift_u64;
extern const loom_b200::KernelEntry loom_b200_entry_rsqrt_f32;
extern const loom_b200::KernelEntry loom_b200_entry_sct_inv_u32;
extern const loom_b200::KernelEntry loom_b200_entry_sin_cos_f32;
extern const loom_b200::KernelEntry loom_b200_entry_slt_inv_u32;
extern const loom_b200::KernelEntry loom_b200_entry_sphere_pt_f32;
extern const loom_b200::KernelEntry loom_b200_entry_sqrt_f32;
extern const loom_b200::KernelEntry loom_b200_entry_threefry_u32;
extern const loom_b200::KernelEntry loom_b200_entry_trunc_f32;
extern const loom_b200::KernelEntry loom_b200_entry_union_cmov_f32;
extern const loom_b200::KernelEntry loom_b200_entry_union_cmov_f64;
extern const loom_b200::KernelEntry loom_b200_entry_union_f32;
extern const loom_b200::KernelEntry loom_b200_entry_union_f64;

namespace loom_b200 {
const KernelEntry* const kRegistry[] = {
    &loom_b200_entry_abs_f32,
    &loom_b200_entry_arithmetic_f32,
    &loom_b200_entry_arithmetic_f64,
    &loom_b200_entry_bit_and_u32,
    &loom_b200_entry_bit_not_u32,
    &loom_b200_entry_bit_not_u8,
    &loom_b200_entry_bit_or_u64,
    &loom_b200_entry_bit_xor_u16,
    &loom_b200_entry_bool_and_u32,
    &loom_b200_entry_bool_not_u8,
    &loom_b200_entry_bool_or_u64,
    &loom_b200_entry_bump_u32,
    &loom_b200_entry_canonical_f32,
    &loom_b200_entry_ceilfloor_f32,
    &loom_b200_entry_collatz_u64,
    &loom_b200_entry_cross_f32,
    &loom_b200_entry_fac_u32,
    &loom_b200_entry_fac_u64,
    &loom_b200_entry_fib_u32,
    &loom_b200_entry_fib_u64,
    &loom_b200_entry_increment_i16,
    &loom_b200_entry_increment_i32,
    &loom_b200_entry_increment_u64,
    &loom_b200_entry_increment_u8,
    &loom_b200_entry_jmp4_f32,
    &loom_b200_entry_jmp4_u16,
    &loom_b200_entry_jmp4_u64,
    &loom_b200_entry_lshift_u16,
    &loom_b200_entry_lshift_u32,
    &loom_b200_entry_lshift_u64,
    &loom_b200_entry_minmax_f32,
    &loom_b200_entry_minmax_f64,
    &loom_b200_entry_norm_f32,
    &loom_b200_entry_primary_const_256,
    &loom_b200_entry_primary_const_b20_256,
    &loom_b200_entry_pt2_const_40,
    &loom_b200_entry_pt2_const_512,
    &loom_b200_entry_pt_const_40,
    &loom_b200_entry_pt_const_512,
    &loom_b200_entry_rotl32_u32,
    &loom_b200_entry_rshift_u16,
    &loom_b200_entry_rshift_u32,
    &loom_b200_entry_rshift_u64,
    &loom_b200_entry_rsqrt_f32,
    &loom_b200_entry_sct_inv_u32,
    &loom_b200_entry_sin_cos_f32,
    &loom_b200_entry_slt_inv_u32,
    &loom_b200_entry_sphere_pt_f32,
    &loom_b200_entry_sqrt_f32,
    &loom_b200_entry_threefry_u32,
    &loom_b200_entry_trunc_f32,
    &loom_b200_entry_union_cmov_f32,
    &loom_b200_entry_union_cmov_f64,
    &loom_b200_entry_union_f32,
    &loom_b200_entry_union_f64,
};
const int kRegistrySize = 55;
} // namespace loom_b200
