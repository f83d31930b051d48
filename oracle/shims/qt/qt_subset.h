/*
 * qt_subset.h -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * The small part of Qt 5's API that the reference's CPU simulator, model
 * classes and evaluator use (Src/Simulator, Src/Model,
 * Src/Search/evaluatormorphogens.cpp), written over the C++ standard library
 * so that those reference files compile unchanged without Qt.  Only what
 * those files call is here, with the behaviour they rely on:
 *
 *   - QList: an array list (append, at, takeAt, removeOne ...).
 *   - QSet: an ordered set.  Qt's QSet iterates in hash order; the simulation
 *     path only ever sorts what it takes out of a set (modelsimulator.cpp:72-74),
 *     so iteration order does not reach a simulated number.
 *   - QHash / QMap: ordered maps with Qt's operator[] and value() rules.
 *   - QTextStream over a QString: ">> int" skips leading white space and reads
 *     a decimal integer; ">> char" and ">> QChar" read the next character as
 *     it is, and give 0 at the end of the text.  The reference's model parser
 *     asserts that the character after every number is a space
 *     (modelprod.cpp:78-95, modellink.cpp:62-84), which holds only if
 *     character reads do not skip white space.  "<< double" prints 6
 *     significant digits, QTextStream's default.
 *   - QString::toDouble parses the whole string (0 if it is not a number).
 *   - Q_ASSERT counts a failed assertion in qt_subset_assert_failures instead
 *     of aborting, so that a harness can report it as an error.
 */
#ifndef GRN_QT_SUBSET_H_
#define GRN_QT_SUBSET_H_

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

typedef unsigned char uchar;
typedef unsigned int uint;
typedef unsigned int QRgb;
typedef long long qint64;

extern std::atomic<int> qt_subset_assert_failures;
inline void qt_subset_assert_failed(const char *cond, const char *file, int line) {
  ++qt_subset_assert_failures;
  std::fprintf(stderr, "Q_ASSERT failed: %s (%s:%d)\n", cond, file, line);
}
#define Q_ASSERT(cond) ((cond) ? (void)0 : qt_subset_assert_failed(#cond, __FILE__, __LINE__))
#define Q_DISABLE_COPY(Class) \
  Class(const Class &) = delete; \
  Class &operator=(const Class &) = delete;

template <typename T>
inline T qAbs(const T &t) { return t >= 0 ? t : -t; }

template <typename T>
class QList {
 public:
  typedef typename std::vector<T>::iterator iterator;
  typedef typename std::vector<T>::const_iterator const_iterator;

  QList() {}
  int size() const { return static_cast<int>(v_.size()); }
  int count() const { return size(); }
  bool isEmpty() const { return v_.empty(); }
  bool empty() const { return v_.empty(); }
  void clear() { v_.clear(); }
  const T &at(int i) const { return v_[i]; }
  T &operator[](int i) { return v_[i]; }
  const T &operator[](int i) const { return v_[i]; }
  T &first() { return v_.front(); }
  const T &first() const { return v_.front(); }
  T &last() { return v_.back(); }
  const T &last() const { return v_.back(); }
  void append(const T &t) { v_.push_back(t); }
  void append(const QList<T> &l) { v_.insert(v_.end(), l.v_.begin(), l.v_.end()); }
  void prepend(const T &t) { v_.insert(v_.begin(), t); }
  QList &operator<<(const T &t) { append(t); return *this; }
  QList &operator+=(const T &t) { append(t); return *this; }
  QList &operator+=(const QList<T> &l) { append(l); return *this; }
  T takeAt(int i) { T t = v_[i]; v_.erase(v_.begin() + i); return t; }
  T takeFirst() { return takeAt(0); }
  T takeLast() { T t = v_.back(); v_.pop_back(); return t; }
  void removeAt(int i) { v_.erase(v_.begin() + i); }
  bool removeOne(const T &t) {
    auto it = std::find(v_.begin(), v_.end(), t);
    if (it == v_.end()) return false;
    v_.erase(it);
    return true;
  }
  int indexOf(const T &t) const {
    auto it = std::find(v_.begin(), v_.end(), t);
    return it == v_.end() ? -1 : static_cast<int>(it - v_.begin());
  }
  bool contains(const T &t) const { return indexOf(t) >= 0; }
  void swap(int i, int j) { std::swap(v_[i], v_[j]); }
  iterator begin() { return v_.begin(); }
  iterator end() { return v_.end(); }
  const_iterator begin() const { return v_.begin(); }
  const_iterator end() const { return v_.end(); }

 private:
  std::vector<T> v_;
};

template <typename T>
class QVector : public QList<T> {};

template <typename C>
inline void qSort(C &c) { std::sort(c.begin(), c.end()); }

template <typename T>
class QSet {
 public:
  typedef typename std::set<T>::const_iterator const_iterator;

  QSet() {}
  int size() const { return static_cast<int>(s_.size()); }
  bool isEmpty() const { return s_.empty(); }
  void clear() { s_.clear(); }
  bool contains(const T &t) const { return s_.count(t) != 0; }
  void insert(const T &t) { s_.insert(t); }
  bool remove(const T &t) { return s_.erase(t) != 0; }
  QSet &operator+=(const T &t) { s_.insert(t); return *this; }
  QSet &operator<<(const T &t) { s_.insert(t); return *this; }
  QSet &unite(const QSet &o) { s_.insert(o.s_.begin(), o.s_.end()); return *this; }
  QSet &operator+=(const QSet &o) { return unite(o); }
  QSet operator+(const QSet &o) const { QSet r = *this; r.unite(o); return r; }
  QSet &intersect(const QSet &o) {
    std::set<T> r;
    for (const T &t : s_)
      if (o.contains(t)) r.insert(t);
    s_.swap(r);
    return *this;
  }
  QSet &subtract(const QSet &o) {
    for (const T &t : o.s_) s_.erase(t);
    return *this;
  }
  QList<T> toList() const {
    QList<T> l;
    for (const T &t : s_) l.append(t);
    return l;
  }
  const_iterator begin() const { return s_.begin(); }
  const_iterator end() const { return s_.end(); }

 private:
  std::set<T> s_;
};

template <typename T>
class QSetIterator {
 public:
  explicit QSetIterator(const QSet<T> &s) : s_(s), it_(s.begin()) {}
  bool hasNext() const { return it_ != s_.end(); }
  const T &next() { return *it_++; }

 private:
  const QSet<T> &s_;
  typename QSet<T>::const_iterator it_;
};

template <typename K, typename V>
class QMap {
 public:
  V &operator[](const K &k) { return m_[k]; }
  V operator[](const K &k) const { return value(k); }
  V value(const K &k, const V &def = V()) const {
    auto it = m_.find(k);
    return it == m_.end() ? def : it->second;
  }
  bool contains(const K &k) const { return m_.count(k) != 0; }
  int size() const { return static_cast<int>(m_.size()); }
  void clear() { m_.clear(); }

 private:
  std::map<K, V> m_;
};

template <typename K, typename V>
class QHash : public QMap<K, V> {};

template <typename A, typename B>
struct QPair {
  A first;
  B second;
};

class QSize {
 public:
  QSize() : w_(-1), h_(-1) {}
  QSize(int w, int h) : w_(w), h_(h) {}
  int width() const { return w_; }
  int height() const { return h_; }
  bool operator==(const QSize &o) const { return w_ == o.w_ && h_ == o.h_; }
  bool operator!=(const QSize &o) const { return !(*this == o); }

 private:
  int w_, h_;
};

class QPoint {
 public:
  QPoint() : x_(0), y_(0) {}
  QPoint(int x, int y) : x_(x), y_(y) {}
  int x() const { return x_; }
  int y() const { return y_; }

 private:
  int x_, y_;
};

class QPointF {
 public:
  QPointF() : x_(0), y_(0) {}
  QPointF(double x, double y) : x_(x), y_(y) {}
  double x() const { return x_; }
  double y() const { return y_; }
  QPointF operator-(const QPointF &o) const { return QPointF(x_ - o.x_, y_ - o.y_); }
  QPointF operator+(const QPointF &o) const { return QPointF(x_ + o.x_, y_ + o.y_); }
  QPointF operator/(double d) const { return QPointF(x_ / d, y_ / d); }
  QPointF operator*(double d) const { return QPointF(x_ * d, y_ * d); }

 private:
  double x_, y_;
};

class QRect {};
class QColor {};

class QChar {
 public:
  QChar() : c_(0) {}
  QChar(char c) : c_(static_cast<unsigned char>(c)) {}
  QChar(int c) : c_(c) {}
  int unicode() const { return c_; }
  char toLatin1() const { return static_cast<char>(c_); }
  bool isSpace() const { return c_ == ' ' || (c_ >= '\t' && c_ <= '\r'); }
  friend bool operator==(QChar a, QChar b) { return a.c_ == b.c_; }
  friend bool operator!=(QChar a, QChar b) { return a.c_ != b.c_; }

 private:
  int c_;
};

class QString {
 public:
  QString() {}
  QString(const char *s) : s_(s ? s : "") {}
  explicit QString(const std::string &s) : s_(s) {}
  QString &append(QChar c) { s_.push_back(c.toLatin1()); return *this; }
  QString &append(const QString &o) { s_ += o.s_; return *this; }
  int size() const { return static_cast<int>(s_.size()); }
  int length() const { return size(); }
  bool isEmpty() const { return s_.empty(); }
  double toDouble(bool *ok = nullptr) const {
    const char *b = s_.c_str();
    char *e = nullptr;
    double v = std::strtod(b, &e);
    bool good = !s_.empty() && e == b + s_.size();
    if (ok) *ok = good;
    return good ? v : 0.0;
  }
  const std::string &str() const { return s_; }
  std::string &str() { return s_; }
  bool operator==(const QString &o) const { return s_ == o.s_; }

 private:
  std::string s_;
};

struct QIODevice {
  enum OpenModeFlag { ReadOnly = 1, WriteOnly = 2, ReadWrite = 3 };
};

class QTextStream {
 public:
  QTextStream(QString *s, int /*mode*/) : s_(s), pos_(0) {}

  qint64 pos() const { return pos_; }
  bool seek(qint64 p) {
    if (p < 0 || p > static_cast<qint64>(s_->str().size())) return false;
    pos_ = p;
    return true;
  }
  bool atEnd() const { return pos_ >= static_cast<qint64>(s_->str().size()); }

  QTextStream &operator>>(char &c) {
    c = atEnd() ? 0 : s_->str()[static_cast<size_t>(pos_++)];
    return *this;
  }
  QTextStream &operator>>(QChar &c) {
    char ch;
    *this >> ch;
    c = QChar(ch);
    return *this;
  }
  QTextStream &operator>>(int &v) {
    const std::string &s = s_->str();
    size_t p = static_cast<size_t>(pos_);
    while (p < s.size() && QChar(s[p]).isSpace()) ++p;
    size_t q = p;
    if (q < s.size() && (s[q] == '-' || s[q] == '+')) ++q;
    size_t digits = q;
    while (q < s.size() && s[q] >= '0' && s[q] <= '9') ++q;
    v = q > digits ? static_cast<int>(std::strtol(s.substr(p, q - p).c_str(), nullptr, 10)) : 0;
    pos_ = static_cast<qint64>(q > digits ? q : p);
    return *this;
  }

  QTextStream &operator<<(char c) { s_->str().push_back(c); return *this; }
  QTextStream &operator<<(QChar c) { return *this << c.toLatin1(); }
  QTextStream &operator<<(int v) { s_->str() += std::to_string(v); return *this; }
  QTextStream &operator<<(double v) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.6g", v);
    s_->str() += buf;
    return *this;
  }
  QTextStream &operator<<(const char *t) { s_->str() += t; return *this; }
  QTextStream &operator<<(const QString &t) { s_->str() += t.str(); return *this; }

 private:
  QString *s_;
  qint64 pos_;
};

/* Image in QImage::Format_RGB32 / ARGB32: one QRgb (0xAARRGGBB) per pixel,
 * rows (scan lines) top to bottom. */
class QImage {
 public:
  QImage() : w_(0), h_(0) {}
  QImage(int w, int h, const QRgb *px) : w_(w), h_(h), px_(px, px + static_cast<size_t>(w) * h) {}
  int width() const { return w_; }
  int height() const { return h_; }
  const uchar *scanLine(int j) const {
    return reinterpret_cast<const uchar *>(px_.data() + static_cast<size_t>(j) * w_);
  }

 private:
  int w_, h_;
  std::vector<QRgb> px_;
};

class QPixmap {};
class QByteArray {};
class QMutex {
 public:
  void lock() {}
  void unlock() {}
};
class QFile {};

#endif  // GRN_QT_SUBSET_H_
