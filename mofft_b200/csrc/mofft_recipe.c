/* MOFFT_PLAN_V1 plan recipes: reading and writing the text form of a plan.
 *
 * A recipe is one line of single-space separated fields, then "\n" and a NUL
 * (the interchange format of the reference, src/mofft.c:1760-1771; the GPU
 * device family takes the place of the CPU family):
 *
 *   #   field            form
 *   0   magic            "MOFFT_PLAN_V1"
 *   1   build id         64 lowercase hex digits, equal to mofft_build_id()
 *   2   device family    exactly 8 hex digits
 *   3   precision        "f32" or "f64"
 *   4   length           decimal, >= 2
 *   5   direction        "-1" or "1"
 *   6   placement        decimal, 0 (out of place) or 1 (in place)
 *   7   kernel bank      decimal, < MOFFT_KERNEL_BANK_COUNT
 *   8   blocked mask     exactly 16 hex digits, no bit at or above depth - 1
 *   9   direct input     decimal, 0 or 1
 *   10  stage layout     decimal, 0 or 1
 *   11  depth            decimal, 1 .. MOFFT_MAX_STAGES
 *   12+ radices          depth decimals >= 2 whose product is the length
 *
 * Which status a malformed recipe earns is part of the interface (the
 * reference's tests/test_plan_recipe.c:196-241 pins it).  Every check here
 * belongs to one of six ranked tiers; the reader walks the recipe once,
 * keeps the lowest tier that failed, and answers with that tier's status:
 *
 *   FRAME      buffer framing and character set          INVALID_ARGUMENT
 *   SHAPE      field separators and count, magic, id     INCOMPATIBLE_RECIPE
 *   SYNTAX     digits and widths of the header numbers   INVALID_ARGUMENT
 *   PRECISION  precision tag against the caller's type   INCOMPATIBLE_RECIPE
 *   VALUE      ranges, depth, mask, radix chain          INVALID_ARGUMENT
 *   DEVICE     device family, then hardware support      INCOMPATIBLE_RECIPE /
 *                                                        UNSUPPORTED_HARDWARE
 */
#include <stdint.h>
#include <string.h>

#include "mofft_host.h"
#include "mofft_recipe.h"

#ifndef MOFFT_BINARY_ID
#define MOFFT_BINARY_ID "0000000000000000000000000000000000000000000000000000000000000000"
#endif

#define RECIPE_MAGIC "MOFFT_PLAN_V1"
#define HEADER_FIELDS 12
#define MAX_FIELDS (HEADER_FIELDS + MOFFT_MAX_STAGES)

enum tier { FRAME, SHAPE, SYNTAX, PRECISION, VALUE, DEVICE, PASSED };

static const mofft_status tier_status[] = {
    MOFFT_INVALID_ARGUMENT,  MOFFT_INCOMPATIBLE_RECIPE, MOFFT_INVALID_ARGUMENT,
    MOFFT_INCOMPATIBLE_RECIPE, MOFFT_INVALID_ARGUMENT,
};

typedef enum { F_MAGIC, F_BUILD, F_HEX, F_TAG, F_DECIMAL, F_SIGN } field_form;

/* Form of each header field, its fixed width (hex fields) and the largest
 * value it may hold (decimal fields; checked in the VALUE tier). */
typedef struct {
  field_form form;
  unsigned width;
  uint64_t max;
} field_rule;

static const field_rule header_rules[HEADER_FIELDS] = {
    {F_MAGIC, 0, 0},
    {F_BUILD, 64, 0},
    {F_HEX, 8, 0},
    {F_TAG, 0, 0},
    {F_DECIMAL, 0, UINT64_MAX},
    {F_SIGN, 0, 0},
    {F_DECIMAL, 0, MOFFT_IN_PLACE},
    {F_DECIMAL, 0, MOFFT_KERNEL_BANK_COUNT - 1},
    {F_HEX, 16, 0},
    {F_DECIMAL, 0, 1},
    {F_DECIMAL, 0, MOFFT_STAGE_LAYOUT_SECTION},
    {F_DECIMAL, 0, MOFFT_MAX_STAGES},
};

/* Radix fields: decimal, at most INT32_MAX; a malformed radix is a VALUE
 * failure (the chain is validated after the precision tag). */
static const field_rule radix_rule = {F_DECIMAL, 0, INT32_MAX};

typedef struct {
  enum tier worst; /* lowest failing tier seen so far */
  uint64_t value[MAX_FIELDS];
  size_t fields;
  int negative_direction;
} reader;

static void fail(reader *r, enum tier t) {
  if (t < r->worst) r->worst = t;
}

static int hex_digit(char ch) {
  if (ch >= '0' && ch <= '9') return ch - '0';
  if (ch >= 'a' && ch <= 'f') return ch - 'a' + 10;
  if (ch >= 'A' && ch <= 'F') return ch - 'A' + 10;
  return -1;
}

static int is_lower_hex_id(const char *s, size_t len) {
  if (len != 64) return 0;
  for (size_t i = 0; i < len; ++i)
    if (!((s[i] >= '0' && s[i] <= '9') || (s[i] >= 'a' && s[i] <= 'f'))) return 0;
  return 1;
}

/* Decimal digits -> value; 0 on an empty field, a non-digit or overflow. */
static int read_decimal(const char *s, size_t len, uint64_t *out) {
  if (len == 0) return 0;
  uint64_t v = 0;
  for (size_t i = 0; i < len; ++i) {
    if (s[i] < '0' || s[i] > '9') return 0;
    const uint64_t d = (uint64_t)(s[i] - '0');
    if (v > (UINT64_MAX - d) / 10) return 0;
    v = v * 10 + d;
  }
  *out = v;
  return 1;
}

static int field_is(const char *s, size_t len, const char *word) {
  return strlen(word) == len && memcmp(s, word, len) == 0;
}

static void check_field(reader *r, size_t index, const char *s, size_t len,
                        int precision_bits) {
  const int header = index < HEADER_FIELDS;
  const field_rule *rule = header ? &header_rules[index] : &radix_rule;
  const enum tier syntax_tier = header ? SYNTAX : VALUE;
  uint64_t v = 0;
  switch (rule->form) {
    case F_MAGIC:
      if (!field_is(s, len, RECIPE_MAGIC)) fail(r, SHAPE);
      break;
    case F_BUILD:
      if (!is_lower_hex_id(MOFFT_BINARY_ID, strlen(MOFFT_BINARY_ID)) ||
          !field_is(s, len, MOFFT_BINARY_ID))
        fail(r, SHAPE);
      break;
    case F_HEX:
      if (len != rule->width) {
        fail(r, syntax_tier);
        break;
      }
      for (size_t i = 0; i < len; ++i) {
        const int d = hex_digit(s[i]);
        if (d < 0) {
          fail(r, syntax_tier);
          break;
        }
        v = (v << 4) | (uint64_t)d;
      }
      break;
    case F_TAG:
      if (!field_is(s, len, precision_bits == 64 ? "f64" : "f32")) fail(r, PRECISION);
      break;
    case F_SIGN:
      if (field_is(s, len, "-1"))
        r->negative_direction = 1;
      else if (!field_is(s, len, "1"))
        fail(r, VALUE);
      break;
    case F_DECIMAL:
      if (!read_decimal(s, len, &v))
        fail(r, syntax_tier);
      else if (v > rule->max)
        fail(r, VALUE);
      break;
  }
  r->value[index] = v;
}

/* Checks that need every field: the depth against the field count, the
 * blocked mask against the depth, and the radix chain against the length. */
static void check_chain(reader *r) {
  const uint64_t length = r->value[4], mask = r->value[8], depth = r->value[11];
  if (length < 2 || depth == 0 || r->fields != HEADER_FIELDS + depth) {
    fail(r, VALUE);
    return;
  }
  if (depth - 1 < 64 && (mask >> (depth - 1)) != 0) fail(r, VALUE);
  uint64_t rest = length;
  for (uint64_t i = 0; i < depth; ++i) {
    const uint64_t radix = r->value[HEADER_FIELDS + i];
    if (radix < 2 || rest % radix != 0) {
      fail(r, VALUE);
      return;
    }
    rest /= radix;
  }
  if (rest != 1) fail(r, VALUE);
}

mofft_status mofft_recipe_read(const char *recipe, size_t size, int precision_bits,
                               mofft_recipe *out) {
  /* FRAME: a NUL-terminated line of printable ASCII, no blank at its end. */
  if (!recipe || size < 2 || size > MOFFT_RECIPE_MAX_BYTES || recipe[size - 1] != '\0' ||
      recipe[size - 2] != '\n' || memchr(recipe, '\0', size - 1) != NULL)
    return MOFFT_INVALID_ARGUMENT;
  const size_t body = size - 2;
  for (size_t i = 0; i < body; ++i)
    if ((unsigned char)recipe[i] < 32 || (unsigned char)recipe[i] > 126)
      return MOFFT_INVALID_ARGUMENT;
  if (body > 1 && recipe[body - 1] == ' ') return MOFFT_INVALID_ARGUMENT;

  reader r;
  memset(&r, 0, sizeof(r));
  r.worst = PASSED;
  const char *p = recipe, *end = recipe + body;
  for (;;) {
    if (r.fields == MAX_FIELDS) {
      fail(&r, SHAPE);
      break;
    }
    const char *q = memchr(p, ' ', (size_t)(end - p));
    if (!q) q = end;
    check_field(&r, r.fields++, p, (size_t)(q - p), precision_bits);
    if (q == end || q + 1 == end) break;
    if (q[1] == ' ') { /* an empty field between two blanks */
      fail(&r, SHAPE);
      break;
    }
    p = q + 1;
  }
  if (r.fields <= HEADER_FIELDS)
    fail(&r, SHAPE);
  else
    check_chain(&r);
  if (r.worst != PASSED) return tier_status[r.worst];

  /* DEVICE: only a recipe that passed every other tier reaches the GPU. */
  uint32_t family = 0;
  if (!mofft_device_family(&family) || family != (uint32_t)r.value[2])
    return MOFFT_INCOMPATIBLE_RECIPE;
  if (!mofft_hardware_supports(precision_bits)) return MOFFT_UNSUPPORTED_HARDWARE;

  out->family = (uint32_t)r.value[2];
  out->length = (size_t)r.value[4];
  out->direction = r.negative_direction ? MOFFT_FORWARD : MOFFT_BACKWARD;
  out->placement = (mofft_placement)r.value[6];
  out->bank = (unsigned)r.value[7];
  out->mask = r.value[8];
  out->direct_input = (int)r.value[9];
  out->layout = (mofft_stage_layout)r.value[10];
  out->depth = (int)r.value[11];
  for (int i = 0; i < out->depth; ++i) out->radices[i] = (int)r.value[HEADER_FIELDS + i];
  return MOFFT_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* writer                                                                    */
/* ------------------------------------------------------------------------ */

typedef struct {
  char text[MOFFT_RECIPE_MAX_BYTES];
  size_t len;
  int overflow;
} line_buffer;

static void put_char(line_buffer *b, char ch) {
  if (b->len + 1 >= sizeof(b->text)) {
    b->overflow = 1;
    return;
  }
  b->text[b->len++] = ch;
}

static void put_text(line_buffer *b, const char *s) {
  while (*s) put_char(b, *s++);
}

static void put_unsigned(line_buffer *b, uint64_t v) {
  char digits[20];
  int n = 0;
  do {
    digits[n++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  while (n) put_char(b, digits[--n]);
}

static void put_signed(line_buffer *b, long long v) {
  if (v < 0) {
    put_char(b, '-');
    put_unsigned(b, (uint64_t)(-(v + 1)) + 1);
  } else {
    put_unsigned(b, (uint64_t)v);
  }
}

static void put_hex(line_buffer *b, uint64_t v, unsigned width) {
  static const char digits[] = "0123456789abcdef";
  for (unsigned i = width; i-- > 0;) put_char(b, digits[(v >> (4 * i)) & 15]);
}

mofft_status mofft_recipe_write(const mofft_core *c, char *buffer, size_t capacity,
                                size_t *required) {
  if (!c || !required) return MOFFT_INVALID_ARGUMENT;
  uint32_t family = 0;
  if (!mofft_device_family(&family) ||
      !is_lower_hex_id(MOFFT_BINARY_ID, strlen(MOFFT_BINARY_ID)))
    return MOFFT_UNSUPPORTED_HARDWARE;
  line_buffer b;
  b.len = 0;
  b.overflow = 0;
  put_text(&b, RECIPE_MAGIC " " MOFFT_BINARY_ID " ");
  put_hex(&b, family, 8);
  put_text(&b, c->precision_bits == 64 ? " f64 " : " f32 ");
  put_unsigned(&b, c->length);
  put_char(&b, ' ');
  put_signed(&b, c->direction);
  put_char(&b, ' ');
  put_unsigned(&b, (uint64_t)c->placement);
  put_char(&b, ' ');
  put_unsigned(&b, c->kernel_bank);
  put_char(&b, ' ');
  put_hex(&b, c->blocked_transpose_mask, 16);
  put_char(&b, ' ');
  put_unsigned(&b, (uint64_t)c->direct_input);
  put_char(&b, ' ');
  put_unsigned(&b, (uint64_t)c->stage_layout);
  put_char(&b, ' ');
  put_unsigned(&b, (uint64_t)c->depth);
  for (int i = 0; i < c->depth; ++i) {
    put_char(&b, ' ');
    put_unsigned(&b, (uint64_t)c->factors[i]);
  }
  put_char(&b, '\n');
  if (b.overflow) return MOFFT_INTERNAL_ERROR;
  b.text[b.len] = '\0';
  *required = b.len + 1;
  if (!buffer) return capacity == 0 ? MOFFT_SUCCESS : MOFFT_INVALID_ARGUMENT;
  if (capacity < *required) return MOFFT_BUFFER_TOO_SMALL;
  memcpy(buffer, b.text, *required);
  return MOFFT_SUCCESS;
}
