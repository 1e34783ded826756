/* loom_interp.c — CPU restatement of Loom's scalar backend for the text IR.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle that tests/, smoke() and bench.py's
 * cpu_baseline leg check the CUDA engines against.  The product never links
 * or calls it.
 *
 * It runs one Loom thread at a time exactly as vm::bse does
 * (Loom src/vm/bse.hpp:400-649):
 *   - set_inputs writes the input variables, PC = 0          (bse.hpp:95-106)
 *   - block b runs its statements in order: Compute stores
 *     Op(get_value(args)...) into Dst                          (core.hpp:740-750)
 *   - Jump sets PC to the target; ParmJump reads its variable and
 *     dispatches like threaded_dispatch: 2 labels -> non-zero picks the
 *     second (bse.hpp:180-185), more labels -> switch, values outside the
 *     table end the thread (no case matches, bse.hpp:186-249)
 *   - HALT ends the thread; outputs are read from the output variables
 *                                                            (bse.hpp:108-115)
 * Registers are raw bits; a typed view reads or writes the low bytes, which
 * is Loom's Union punning (src/common/union.hpp).  Operand semantics are
 * those of the std:: functors and loom::vm::ops (src/vm/operators.hpp):
 * arguments are converted to the functor's operand type with C++ integer
 * promotion, the functor's result type is kept, and the result is converted
 * to the destination type.  Built with -ffp-contract=off so float arithmetic
 * is rounded per operation.
 *
 * C ABI (see oracle/oracle.py):
 *   void* li_load(const char* ir_text)               parse; NULL on error
 *   const char* li_error(void)
 *   int   li_run(void* k, const void* const* in, void* const* out,
 *                uint64_t n, uint64_t max_steps, uint64_t* instr_counts,
 *                const uint32_t* table)      table: words of the tab op
 *   void  li_free(void* k)
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum
{
    T_B8,
    T_I8,
    T_U8,
    T_I16,
    T_U16,
    T_I32,
    T_U32,
    T_I64,
    T_U64,
    T_F32,
    T_F64,
    T_NONE
};

static const char* const TNAMES[] = {"b8", "i8", "u8", "i16", "u16", "i32",
                                     "u32", "i64", "u64", "f32", "f64"};
static const int TBYTES[] = {1, 1, 1, 2, 2, 4, 4, 8, 8, 4, 8};

static int
is_float(int t)
{
    return t == T_F32 || t == T_F64;
}
static int
is_signed(int t)
{
    return t == T_I8 || t == T_I16 || t == T_I32 || t == T_I64;
}

enum
{
    OP_MOV,
    OP_CMOV,
    OP_FMA,
    OP_FMS,
    OP_ASSERT_FP,
    OP_ADD,
    OP_SUB,
    OP_MUL,
    OP_DIV,
    OP_MOD,
    OP_NEG,
    OP_EQ,
    OP_NE,
    OP_GT,
    OP_LT,
    OP_GE,
    OP_LE,
    OP_LAND,
    OP_LOR,
    OP_LNOT,
    OP_BAND,
    OP_BOR,
    OP_BXOR,
    OP_BNOT,
    OP_SHL,
    OP_SHR,
    OP_ABS,
    OP_RSQRT,
    OP_MAX,
    OP_MIN,
    OP_ROUND,
    OP_CEIL,
    OP_FLOOR,
    OP_TRUNC,
    OP_SIN,
    OP_COS,
    OP_SQRT,
    OP_COPYSIGN,
    OP_SCT,
    OP_SLT,
    OP_PACC,
    OP_TAB,
    OP_COUNT
};

static const char* const OPNAMES[] = {
    "mov",   "cmov", "fma",   "fms",  "assert_fp", "add",   "sub",  "mul",
    "div",   "mod",  "neg",   "eq",   "ne",        "gt",    "lt",   "ge",
    "le",    "land", "lor",   "lnot", "band",      "bor",   "bxor", "bnot",
    "shl",   "shr",  "abs",   "rsqrt", "max",      "min",   "round", "ceil",
    "floor", "trunc", "sin",  "cos",  "sqrt",      "copysign", "sct", "slt",
    "pacc",  "tab"};

/* typed value */
typedef struct
{
    int t;
    union
    {
        uint64_t u;
        int64_t  i;
        float    f;
        double   d;
    } v;
} val;

typedef struct
{
    int      t;
    int      reg; /* -1: literal */
    uint64_t bits;
} operand;

typedef struct
{
    int      kind; /* 0 compute, 1 jump, 2 parmjump */
    int      op;
    int      ot[4]; /* operand types of the functor (T_NONE if generic) */
    int      cmp, acc; /* pacc */
    operand  dst;
    int      nargs;
    operand* args;
    int      nconsts;
    operand* consts;
    int      ntargets;
    int*     targets;
} instr;

typedef struct
{
    int    ninstr;
    instr* ins;
} block;

typedef struct
{
    int      nregs;
    int*     rbytes;
    int      nin, nout;
    int*     in_reg;
    int*     in_t;
    int*     out_reg;
    int*     out_t;
    int      nblocks;
    block*   blocks;
} kernel;

static char g_err[256];

const char*
li_error(void)
{
    return g_err;
}

static int
parse_type(const char* s)
{
    for(int i = 0; i < T_NONE; ++i)
        if(strcmp(s, TNAMES[i]) == 0) return i;
    return -1;
}

static int
parse_operand(const char* tok, operand* o)
{
    char tbuf[8];
    if(tok[0] == 'r')
    {
        int reg;
        if(sscanf(tok + 1, "%d:%7s", &reg, tbuf) != 2) return -1;
        o->reg  = reg;
        o->t    = parse_type(tbuf);
        o->bits = 0;
        return o->t < 0 ? -1 : 0;
    }
    if(tok[0] == 'k')
    {
        const char* colon = strchr(tok, ':');
        if(!colon || colon - tok - 1 >= (long)sizeof(tbuf)) return -1;
        memcpy(tbuf, tok + 1, colon - tok - 1);
        tbuf[colon - tok - 1] = 0;
        o->reg  = -1;
        o->t    = parse_type(tbuf);
        o->bits = strtoull(colon + 1, NULL, 16);
        return o->t < 0 ? -1 : 0;
    }
    return -1;
}

static int
cmp_code(const char* s)
{
    const char* names[] = {"eq", "ne", "gt", "lt", "ge", "le"};
    for(int i = 0; i < 6; ++i)
        if(strcmp(s, names[i]) == 0) return OP_EQ + i;
    return -1;
}

void li_free(void* p);

/* tokenise one line in place */
static int
split(char* line, char** tok, int max)
{
    int n = 0;
    for(char* s = strtok(line, " \t\r\n"); s && n < max; s = strtok(NULL, " \t\r\n"))
        tok[n++] = s;
    return n;
}

void*
li_load(const char* text)
{
    kernel* k = calloc(1, sizeof(kernel));
    char*   buf = strdup(text);
    int     cur = -1;
    int     ok  = 1;
    /* first pass: counts */
    int nregs = 0, nin = 0, nout = 0, nblocks = 0;
    for(const char* p = text; *p;)
    {
        if(!strncmp(p, "reg ", 4)) nregs++;
        if(!strncmp(p, "input ", 6)) nin++;
        if(!strncmp(p, "output ", 7)) nout++;
        if(!strncmp(p, "block ", 6)) nblocks++;
        const char* nl = strchr(p, '\n');
        if(!nl) break;
        p = nl + 1;
    }
    k->nregs   = nregs;
    k->rbytes  = calloc(nregs + 1, sizeof(int));
    k->in_reg  = calloc(nin + 1, sizeof(int));
    k->in_t    = calloc(nin + 1, sizeof(int));
    k->out_reg = calloc(nout + 1, sizeof(int));
    k->out_t   = calloc(nout + 1, sizeof(int));
    k->blocks  = calloc(nblocks + 1, sizeof(block));
    k->nblocks = nblocks;
    char* save = NULL;
    for(char* line = strtok_r(buf, "\n", &save); line && ok;
        line = strtok_r(NULL, "\n", &save))
    {
        char  lcopy[4096];
        char* tok[520];
        strncpy(lcopy, line, sizeof(lcopy) - 1);
        lcopy[sizeof(lcopy) - 1] = 0;
        int nt = split(lcopy, tok, 520);
        if(nt == 0) continue;
        if(!strcmp(tok[0], "reg"))
            k->rbytes[atoi(tok[1])] = atoi(tok[3]);
        else if(!strcmp(tok[0], "input"))
        {
            k->in_reg[k->nin] = atoi(tok[1]);
            k->in_t[k->nin++] = parse_type(tok[2]);
        }
        else if(!strcmp(tok[0], "output"))
        {
            k->out_reg[k->nout] = atoi(tok[1]);
            k->out_t[k->nout++] = parse_type(tok[2]);
        }
        else if(!strcmp(tok[0], "block"))
        {
            cur                    = atoi(tok[1]);
            k->blocks[cur].ninstr  = 0;
            k->blocks[cur].ins     = calloc(atoi(tok[3]) + 1, sizeof(instr));
        }
        else if(!strcmp(tok[0], "i") || !strcmp(tok[0], "j") || !strcmp(tok[0], "p"))
        {
            if(cur < 0)
            {
                ok = 0;
                break;
            }
            instr* in = &k->blocks[cur].ins[k->blocks[cur].ninstr++];
            if(tok[0][0] == 'j')
            {
                in->kind       = 1;
                in->ntargets   = 1;
                in->targets    = calloc(1, sizeof(int));
                in->targets[0] = atoi(tok[1]);
            }
            else if(tok[0][0] == 'p')
            {
                in->kind = 2;
                in->args = calloc(1, sizeof(operand));
                if(parse_operand(tok[1], &in->args[0])) ok = 0;
                in->nargs    = 1;
                in->ntargets = nt - 2;
                in->targets  = calloc(nt, sizeof(int));
                for(int i = 2; i < nt; ++i) in->targets[i - 2] = atoi(tok[i]);
            }
            else
            {
                in->kind = 0;
                in->op   = -1;
                for(int o = 0; o < OP_COUNT; ++o)
                    if(!strcmp(tok[1], OPNAMES[o])) in->op = o;
                if(in->op < 0)
                {
                    snprintf(g_err, sizeof g_err, "unknown op %s", tok[1]);
                    ok = 0;
                    break;
                }
                for(int j = 0; j < 4; ++j) in->ot[j] = T_NONE;
                if(strcmp(tok[2], "-"))
                {
                    char  ots[64];
                    char* sv = NULL;
                    strncpy(ots, tok[2], 63);
                    ots[63] = 0;
                    int j   = 0;
                    for(char* s = strtok_r(ots, ",", &sv); s; s = strtok_r(NULL, ",", &sv), ++j)
                    {
                        if(in->op == OP_PACC && j == 2)
                            in->acc = !strcmp(s, "land") ? OP_LAND : OP_LOR;
                        else if(in->op == OP_PACC && j == 3)
                            in->cmp = cmp_code(s);
                        else if(j < 4)
                            in->ot[j] = parse_type(s);
                    }
                }
                int bar = nt;
                for(int i = 3; i < nt; ++i)
                    if(!strcmp(tok[i], "|")) bar = i;
                if(nt < 4 || bar < 4)
                {
                    snprintf(g_err, sizeof g_err, "malformed instruction");
                    ok = 0;
                    break;
                }
                if(parse_operand(tok[3], &in->dst)) ok = 0;
                in->nargs = bar - 4;
                in->args  = calloc(in->nargs + 1, sizeof(operand));
                for(int i = 0; i < in->nargs; ++i)
                    if(parse_operand(tok[4 + i], &in->args[i])) ok = 0;
                in->nconsts = bar < nt ? nt - bar - 1 : 0;
                in->consts  = calloc(in->nconsts + 1, sizeof(operand));
                for(int i = 0; i < in->nconsts; ++i)
                    if(parse_operand(tok[bar + 1 + i], &in->consts[i])) ok = 0;
            }
        }
    }
    free(buf);
    if(!ok)
    {
        if(!g_err[0]) snprintf(g_err, sizeof g_err, "IR parse error");
        li_free(k);
        return NULL;
    }
    return k;
}

void
li_free(void* p)
{
    kernel* k = p;
    if(!k) return;
    for(int b = 0; b < k->nblocks; ++b)
    {
        for(int i = 0; i < k->blocks[b].ninstr; ++i)
        {
            free(k->blocks[b].ins[i].args);
            free(k->blocks[b].ins[i].consts);
            free(k->blocks[b].ins[i].targets);
        }
        free(k->blocks[b].ins);
    }
    free(k->blocks);
    free(k->rbytes);
    free(k->in_reg);
    free(k->in_t);
    free(k->out_reg);
    free(k->out_t);
    free(k);
}

/* ------------------------------------------------------------ values */
static val
from_bits(int t, uint64_t bits)
{
    val r;
    r.t   = t;
    r.v.u = 0;
    switch(t)
    {
    case T_B8: r.v.u = (bits & 0xff) != 0; break;
    case T_I8: r.v.i = (int8_t)bits; break;
    case T_U8: r.v.u = (uint8_t)bits; break;
    case T_I16: r.v.i = (int16_t)bits; break;
    case T_U16: r.v.u = (uint16_t)bits; break;
    case T_I32: r.v.i = (int32_t)bits; break;
    case T_U32: r.v.u = (uint32_t)bits; break;
    case T_I64: r.v.i = (int64_t)bits; break;
    case T_U64: r.v.u = bits; break;
    case T_F32:
    {
        uint32_t b = (uint32_t)bits;
        memcpy(&r.v.f, &b, 4);
        break;
    }
    case T_F64: memcpy(&r.v.d, &bits, 8); break;
    }
    return r;
}

static uint64_t
to_bits(val x)
{
    uint64_t b = 0;
    switch(x.t)
    {
    case T_F32:
    {
        uint32_t u;
        memcpy(&u, &x.v.f, 4);
        b = u;
        break;
    }
    case T_F64: memcpy(&b, &x.v.d, 8); break;
    default: b = x.v.u; break;
    }
    int nb = TBYTES[x.t];
    return nb == 8 ? b : (b & ((1ull << (8 * nb)) - 1));
}

/* C++ static_cast between arithmetic types */
static val
convert(val x, int t)
{
    if(x.t == t) return x;
    val r;
    r.t   = t;
    r.v.u = 0;
    if(t == T_B8)
    {
        if(x.t == T_F32)
            r.v.u = x.v.f != 0.0f;
        else if(x.t == T_F64)
            r.v.u = x.v.d != 0.0;
        else
            r.v.u = x.v.u != 0;
        return r;
    }
    if(is_float(t))
    {
        double d;
        float  f;
        if(x.t == T_F32)
        {
            f = x.v.f;
            d = x.v.f;
        }
        else if(x.t == T_F64)
        {
            d = x.v.d;
            f = (float)x.v.d;
        }
        else if(is_signed(x.t))
        {
            d = (double)x.v.i;
            f = (float)x.v.i;
        }
        else
        {
            d = (double)x.v.u;
            f = (float)x.v.u;
        }
        if(t == T_F32)
            r.v.f = f;
        else
            r.v.d = d;
        return r;
    }
    /* integer target */
    uint64_t bits;
    if(x.t == T_F32 || x.t == T_F64)
    {
        double d = x.t == T_F32 ? (double)x.v.f : x.v.d;
        if(is_signed(t))
            bits = (uint64_t)(int64_t)d;
        else if(t == T_U64)
            bits = (uint64_t)d;
        else
            bits = (uint64_t)(int64_t)d;
    }
    else
        bits = x.v.u; /* two's complement: i and u share bits */
    return from_bits(t, bits);
}

static val
mk_bool(int b)
{
    val r;
    r.t   = T_B8;
    r.v.u = b != 0;
    return r;
}

static int
truthy(val x)
{
    if(x.t == T_F32) return x.v.f != 0.0f;
    if(x.t == T_F64) return x.v.d != 0.0;
    return x.v.u != 0;
}

static int
compare(int op, val a, val b)
{
    int t = a.t;
    if(t == T_F32)
    {
        float x = a.v.f, y = b.v.f;
        switch(op)
        {
        case OP_EQ: return x == y;
        case OP_NE: return x != y;
        case OP_GT: return x > y;
        case OP_LT: return x < y;
        case OP_GE: return x >= y;
        default: return x <= y;
        }
    }
    if(t == T_F64)
    {
        double x = a.v.d, y = b.v.d;
        switch(op)
        {
        case OP_EQ: return x == y;
        case OP_NE: return x != y;
        case OP_GT: return x > y;
        case OP_LT: return x < y;
        case OP_GE: return x >= y;
        default: return x <= y;
        }
    }
    if(is_signed(t))
    {
        int64_t x = a.v.i, y = b.v.i;
        switch(op)
        {
        case OP_EQ: return x == y;
        case OP_NE: return x != y;
        case OP_GT: return x > y;
        case OP_LT: return x < y;
        case OP_GE: return x >= y;
        default: return x <= y;
        }
    }
    uint64_t x = a.v.u, y = b.v.u;
    switch(op)
    {
    case OP_EQ: return x == y;
    case OP_NE: return x != y;
    case OP_GT: return x > y;
    case OP_LT: return x < y;
    case OP_GE: return x >= y;
    default: return x <= y;
    }
}

/* integer binary op at operand type t, with C++ promotion: results wrap to
 * the width of t (as std::plus<T> etc. return T) */
static val
int_binop(int op, val a, val b, int t)
{
    uint64_t r  = 0;
    int      sg = is_signed(t) || TBYTES[t] < 4; /* promoted to int */
    /* values sign- or zero-extended to 64 bits */
    int64_t  xi = a.v.i, yi = b.v.i;
    uint64_t xu = a.v.u, yu = b.v.u;
    switch(op)
    {
    case OP_ADD: r = xu + yu; break;
    case OP_SUB: r = xu - yu; break;
    case OP_MUL: r = xu * yu; break;
    case OP_DIV:
        if(sg)
            r = yi ? (uint64_t)(xi / yi) : 0;
        else
            r = yu ? xu / yu : 0;
        break;
    case OP_MOD:
        if(sg)
            r = yi ? (uint64_t)(xi % yi) : 0;
        else
            r = yu ? xu % yu : 0;
        break;
    case OP_BAND: r = xu & yu; break;
    case OP_BOR: r = xu | yu; break;
    case OP_BXOR: r = xu ^ yu; break;
    case OP_SHL: r = yu < 64 ? xu << yu : 0; break;
    case OP_SHR:
        if(is_signed(t))
            r = yu < 64 ? (uint64_t)(xi >> yu) : (uint64_t)(xi >> 63);
        else
            r = yu < 64 ? xu >> yu : 0;
        break;
    }
    return from_bits(t, r);
}

static val
read_op(const kernel* k, const uint64_t* R, const operand* o)
{
    (void)k;
    if(o->reg < 0) return from_bits(o->t, o->bits);
    return from_bits(o->t, R[o->reg]);
}

static void
write_reg(const kernel* k, uint64_t* R, const operand* dst, val x)
{
    x              = convert(x, dst->t);
    uint64_t bits  = to_bits(x);
    int      nb    = TBYTES[dst->t];
    int      rb    = k->rbytes[dst->reg];
    uint64_t mask  = nb == 8 ? ~0ull : ((1ull << (8 * nb)) - 1);
    if(nb >= rb)
        R[dst->reg] = bits;
    else
        R[dst->reg] = (R[dst->reg] & ~mask) | bits;
}

static val
fp_unary(int op, val a)
{
    val r = a;
    if(a.t == T_F32)
    {
        float x = a.v.f;
        switch(op)
        {
        case OP_ROUND: r.v.f = roundf(x); break;
        case OP_CEIL: r.v.f = ceilf(x); break;
        case OP_FLOOR: r.v.f = floorf(x); break;
        case OP_TRUNC: r.v.f = truncf(x); break;
        case OP_SIN: r.v.f = sinf(x); break;
        case OP_COS: r.v.f = cosf(x); break;
        case OP_SQRT: r.v.f = sqrtf(x); break;
        case OP_RSQRT: r.v.f = 1.0f / sqrtf(x); break;
        case OP_ABS: r.v.f = fabsf(x); break;
        case OP_NEG: r.v.f = -x; break;
        }
    }
    else
    {
        double x = a.v.d;
        switch(op)
        {
        case OP_ROUND: r.v.d = round(x); break;
        case OP_CEIL: r.v.d = ceil(x); break;
        case OP_FLOOR: r.v.d = floor(x); break;
        case OP_TRUNC: r.v.d = trunc(x); break;
        case OP_SIN: r.v.d = sin(x); break;
        case OP_COS: r.v.d = cos(x); break;
        case OP_SQRT: r.v.d = sqrt(x); break;
        case OP_RSQRT: r.v.d = 1.0 / sqrt(x); break;
        case OP_ABS: r.v.d = fabs(x); break;
        case OP_NEG: r.v.d = -x; break;
        }
    }
    return r;
}

static val
fp_binop(int op, val a, val b)
{
    val r = a;
    if(a.t == T_F32)
    {
        float x = a.v.f, y = b.v.f;
        switch(op)
        {
        case OP_ADD: r.v.f = x + y; break;
        case OP_SUB: r.v.f = x - y; break;
        case OP_MUL: r.v.f = x * y; break;
        case OP_DIV: r.v.f = x / y; break;
        case OP_MAX: r.v.f = (x < y) ? y : x; break;
        case OP_MIN: r.v.f = (y < x) ? y : x; break;
        case OP_COPYSIGN: r.v.f = copysignf(x, y); break;
        }
    }
    else
    {
        double x = a.v.d, y = b.v.d;
        switch(op)
        {
        case OP_ADD: r.v.d = x + y; break;
        case OP_SUB: r.v.d = x - y; break;
        case OP_MUL: r.v.d = x * y; break;
        case OP_DIV: r.v.d = x / y; break;
        case OP_MAX: r.v.d = (x < y) ? y : x; break;
        case OP_MIN: r.v.d = (y < x) ? y : x; break;
        case OP_COPYSIGN: r.v.d = copysign(x, y); break;
        }
    }
    return r;
}

/* one Compute statement; `table` is the word table of the tab extension */
static int
compute(const kernel* k, uint64_t* R, const instr* in, const uint32_t* table)
{
    val a[8];
    int na = in->nargs < 8 ? in->nargs : 8;
    for(int i = 0; i < na; ++i) a[i] = read_op(k, R, &in->args[i]);
    int t = in->ot[0];
    val r;
    switch(in->op)
    {
    case OP_MOV: r = a[0]; break;
    case OP_ASSERT_FP: r = a[0]; break;
    case OP_CMOV: r = truthy(a[0]) ? a[1] : a[2]; break;
    case OP_FMA:
    case OP_FMS:
        r = a[0];
        if(a[0].t == T_F32)
            r.v.f = fmaf(a[0].v.f, a[1].v.f, in->op == OP_FMA ? a[2].v.f : -a[2].v.f);
        else
            r.v.d = fma(a[0].v.d, a[1].v.d, in->op == OP_FMA ? a[2].v.d : -a[2].v.d);
        break;
    case OP_EQ:
    case OP_NE:
    case OP_GT:
    case OP_LT:
    case OP_GE:
    case OP_LE: r = mk_bool(compare(in->op, convert(a[0], t), convert(a[1], t))); break;
    case OP_LAND: r = mk_bool(truthy(convert(a[0], t)) && truthy(convert(a[1], t))); break;
    case OP_LOR: r = mk_bool(truthy(convert(a[0], t)) || truthy(convert(a[1], t))); break;
    case OP_LNOT: r = mk_bool(!truthy(convert(a[0], t))); break;
    case OP_NEG:
    case OP_BNOT:
    case OP_ABS:
    {
        val x = convert(a[0], t);
        if(is_float(t))
            r = fp_unary(in->op, x);
        else
        {
            uint64_t u = x.v.u;
            if(in->op == OP_NEG)
                u = 0 - u;
            else if(in->op == OP_BNOT)
                u = ~u;
            else if(is_signed(t) && x.v.i < 0)
                u = (uint64_t)(-x.v.i);
            r = from_bits(t, u);
        }
        break;
    }
    case OP_ADD:
    case OP_SUB:
    case OP_MUL:
    case OP_DIV:
    case OP_MOD:
    case OP_BAND:
    case OP_BOR:
    case OP_BXOR:
    case OP_SHL:
    case OP_SHR:
    {
        val x = convert(a[0], t), y = convert(a[1], t);
        r = is_float(t) ? fp_binop(in->op, x, y) : int_binop(in->op, x, y, t);
        break;
    }
    case OP_MAX:
    case OP_MIN:
    {
        val x = convert(a[0], t), y = convert(a[1], t);
        if(is_float(t))
            r = fp_binop(in->op, x, y);
        else
        {
            int lt = in->op == OP_MAX ? compare(OP_LT, x, y) : compare(OP_LT, y, x);
            r      = lt ? y : x;
        }
        break;
    }
    case OP_COPYSIGN: r = fp_binop(OP_COPYSIGN, convert(a[0], t), convert(a[1], t)); break;
    case OP_ROUND:
    case OP_CEIL:
    case OP_FLOOR:
    case OP_TRUNC:
    case OP_SIN:
    case OP_COS:
    case OP_SQRT:
    case OP_RSQRT: r = fp_unary(in->op, convert(a[0], t)); break;
    case OP_SCT:
    {
        val      i  = convert(a[0], in->ot[1]);
        uint64_t ix = i.v.u;
        if(ix >= (uint64_t)in->nconsts) ix = in->nconsts - 1;
        r = convert(from_bits(in->consts[ix].t, in->consts[ix].bits), t);
        break;
    }
    case OP_SLT:
    {
        val      i  = convert(a[0], in->ot[1]);
        uint64_t ix = i.v.u;
        if(ix >= (uint64_t)(na - 1)) ix = na - 2;
        r = convert(a[1 + ix], t);
        break;
    }
    case OP_TAB:
    {
        /* word idx of the table, read as the op's type (a 32-bit type) */
        uint64_t idx = convert(a[0], T_U32).v.u;
        r = from_bits(t, table ? table[idx] : 0u);
        break;
    }
    case OP_PACC:
    {
        int it = in->ot[1];
        int c  = compare(in->cmp, convert(a[1], t), convert(a[2], t));
        int p  = truthy(convert(a[0], it));
        int q  = truthy(convert(mk_bool(c), it));
        r      = convert(mk_bool(in->acc == OP_LAND ? (p && q) : (p || q)), it);
        break;
    }
    default: return -1;
    }
    write_reg(k, R, &in->dst, r);
    return 0;
}

/* Runs threads [0, n).  Returns 0, or -1 when a thread exceeded max_steps
 * block executions.  instr_counts (optional) receives per-thread executed
 * instruction counts. */
int
li_run(void*              kp,
       const void* const* in,
       void* const*       out,
       uint64_t           n,
       uint64_t           max_steps,
       uint64_t*          instr_counts,
       const uint32_t*    table)
{
    const kernel* k      = kp;
    uint64_t*     R      = calloc(k->nregs + 1, sizeof(uint64_t));
    int           status = 0;
    for(uint64_t t = 0; t < n; ++t)
    {
        memset(R, 0, (k->nregs + 1) * sizeof(uint64_t));
        for(int i = 0; i < k->nin; ++i)
        {
            int      ty = k->in_t[i];
            uint64_t bits = 0;
            if(in[i])
                memcpy(&bits, (const char*)in[i] + t * TBYTES[ty], TBYTES[ty]);
            else
                bits = to_bits(convert(from_bits(T_U64, t), ty));
            operand dst = {ty, k->in_reg[i], 0};
            write_reg(k, R, &dst, from_bits(ty, bits));
        }
        int      pc    = 0;
        uint64_t steps = 0, icount = 0;
        while(pc >= 0)
        {
            if(++steps > max_steps)
            {
                status = -1;
                break;
            }
            const block* b    = &k->blocks[pc];
            int          next = -1;
            for(int i = 0; i < b->ninstr; ++i)
            {
                const instr* ins = &b->ins[i];
                ++icount;
                if(ins->kind == 0)
                    compute(k, R, ins, table);
                else if(ins->kind == 1)
                    next = ins->targets[0];
                else
                {
                    val      v  = read_op(k, R, &ins->args[0]);
                    uint64_t ix = v.v.u;
                    if(ins->ntargets == 2)
                        next = ix ? ins->targets[1] : ins->targets[0];
                    else
                        next = ix < (uint64_t)ins->ntargets ? ins->targets[ix] : -1;
                }
            }
            pc = next;
        }
        if(instr_counts) instr_counts[t] = icount;
        for(int j = 0; j < k->nout; ++j)
        {
            int      ty   = k->out_t[j];
            uint64_t bits = to_bits(from_bits(ty, R[k->out_reg[j]]));
            memcpy((char*)out[j] + t * TBYTES[ty], &bits, TBYTES[ty]);
        }
    }
    free(R);
    return status;
}
