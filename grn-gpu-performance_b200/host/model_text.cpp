// model_text.cpp -- the reference's text form of a model, for run files and
// for exchanging models with the reference's tools.
//
// Restates Model operator<< / operator>> (Src/Model/model.cpp:628-706),
// ModelProd's (Src/Model/modelprod.cpp:74-106) and ModelLink's
// (Src/Model/modellink.cpp:56-90):
//   "(" product ("|" product)* "*" [link ("|" link)*] ")"
//   product = label init lim deg dif        (space separated)
//   link    = regulator regulated K n isAnd (isAnd written 1 / 0)
// Doubles are written like QTextStream's default (6 significant digits,
// shortest of fixed / scientific, as printf "%g"); `precision` 17 writes
// them exactly.  Parsing never aborts: malformed text is GRN_ERR_MODEL.

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/grn_gpu.h"

namespace {

void put_double(std::string *out, double v, int precision) {
  char b[64];
  std::snprintf(b, sizeof b, "%.*g", precision, v);
  out->append(b);
}

struct Reader {
  const char *p;
  void skip_spaces() {
    while (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r') ++p;
  }
  bool expect(char c) {
    skip_spaces();
    if (*p != c) return false;
    ++p;
    return true;
  }
  bool peek(char c) {
    skip_spaces();
    return *p == c;
  }
  bool read_int(int32_t *v) {
    skip_spaces();
    char *end = nullptr;
    errno = 0;
    const long x = std::strtol(p, &end, 10);
    if (end == p || errno != 0 || x < INT32_MIN || x > INT32_MAX) return false;
    *v = (int32_t)x;
    p = end;
    return true;
  }
  // A number ends at a space or at one of | * ) (Model::parseDouble).
  bool read_double(double *v) {
    skip_spaces();
    const char *q = p;
    while (*q && *q != ' ' && *q != '|' && *q != '*' && *q != ')') ++q;
    if (q == p) return false;
    std::string tok(p, q);
    char *end = nullptr;
    *v = std::strtod(tok.c_str(), &end);
    if (end != tok.c_str() + tok.size()) return false;
    p = q;
    return true;
  }
};

}  // namespace

extern "C" {

grn_status grn_model_format(const grn_product *products, int n_products, const grn_link *links,
                            int n_links, int precision, char *buf, int buf_len, int *needed) {
  if (n_products < 0 || n_links < 0 || (n_products && !products) || (n_links && !links) ||
      precision < 1 || precision > 17 || buf_len < 0 || (buf_len > 0 && !buf))
    return GRN_ERR_INVALID_ARGUMENT;
  std::string s = "(";
  for (int i = 0; i < n_products; ++i) {
    const grn_product &p = products[i];
    if (i) s += '|';
    s += std::to_string(p.label);
    s += ' ';
    put_double(&s, p.init, precision);
    s += ' ';
    put_double(&s, p.lim, precision);
    s += ' ';
    put_double(&s, p.deg, precision);
    s += ' ';
    put_double(&s, p.dif, precision);
  }
  s += '*';
  for (int i = 0; i < n_links; ++i) {
    const grn_link &l = links[i];
    if (i) s += '|';
    s += std::to_string(l.regulator);
    s += ' ';
    s += std::to_string(l.regulated);
    s += ' ';
    put_double(&s, l.dis_const, precision);
    s += ' ';
    put_double(&s, l.hill_coef, precision);
    s += l.is_and ? " 1" : " 0";
  }
  s += ')';
  if (needed) *needed = (int)s.size() + 1;
  if ((int)s.size() + 1 > buf_len) return GRN_ERR_CAPACITY;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return GRN_OK;
}

grn_status grn_model_parse(const char *text, grn_product *products, int max_products,
                           int *n_products, grn_link *links, int max_links, int *n_links) {
  if (!text || !n_products || !n_links || max_products < 0 || max_links < 0 ||
      (max_products && !products) || (max_links && !links))
    return GRN_ERR_INVALID_ARGUMENT;
  Reader r{text};
  int np = 0, nl = 0;
  if (!r.expect('(')) return GRN_ERR_MODEL;
  // Products up to '*' (the reference reads at least one).
  for (;;) {
    grn_product p{};
    if (!r.read_int(&p.label) || !r.read_double(&p.init) || !r.read_double(&p.lim) ||
        !r.read_double(&p.deg) || !r.read_double(&p.dif))
      return GRN_ERR_MODEL;
    if (np < max_products) products[np] = p;
    ++np;
    if (r.expect('*')) break;
    if (!r.expect('|')) return GRN_ERR_MODEL;
  }
  if (!r.expect(')')) {
    for (;;) {
      grn_link l{};
      int32_t is_and = 0;
      if (!r.read_int(&l.regulator) || !r.read_int(&l.regulated) ||
          !r.read_double(&l.dis_const) || !r.read_double(&l.hill_coef) || !r.read_int(&is_and))
        return GRN_ERR_MODEL;
      l.is_and = is_and != 0;
      if (nl < max_links) links[nl] = l;
      ++nl;
      if (r.expect(')')) break;
      if (!r.expect('|')) return GRN_ERR_MODEL;
    }
  }
  r.skip_spaces();
  if (*r.p != '\0') return GRN_ERR_MODEL;
  *n_products = np;
  *n_links = nl;
  return (np > max_products || nl > max_links) ? GRN_ERR_CAPACITY : GRN_OK;
}

}  // extern "C"
