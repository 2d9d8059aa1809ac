// std-backed stand-ins for the Qt types that the reference's hot-path
// sources name, so that they compile unchanged without Qt for the oracle/_ref
// harness (test infrastructure).  Only what those sources touch is provided;
// GUI, file, network and painting types are empty shells.
#pragma once
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <set>
#include <stack>
#include <cstdint>
#include <map>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

typedef uint8_t quint8;
typedef uint16_t quint16;
typedef uint32_t quint32;
typedef unsigned long long quint64;
typedef int8_t qint8;
typedef int16_t qint16;
typedef int32_t qint32;
typedef long long qint64;
typedef unsigned int uint;
typedef unsigned char uchar;
typedef unsigned short ushort;
typedef double qreal;

template <class T>
inline const T &qMin(const T &a, const T &b) { return (a < b) ? a : b; }
template <class T>
inline const T &qMax(const T &a, const T &b) { return (a < b) ? b : a; }
template <class T>
inline const T &qBound(const T &lo, const T &v, const T &hi) { return qMax(lo, qMin(v, hi)); }
template <class T>
inline T qAbs(const T &v) { return v >= T(0) ? v : -v; }

template <class T>
class QList;
class QChar;

class QString {
 public:
  QString() {}
  QString(const char *s) : s_(s ? s : "") {}
  QString(const std::string &s) : s_(s) {}
  QString(char c) : s_(1, c) {}
  QString(const QChar &c);
  static QString number(double v) {  // format 'g', precision 6 (Qt's defaults)
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%g", v);
    return QString(buf);
  }
  static QString number(int v) { return QString(std::to_string(v)); }
  static QString number(long long v) { return QString(std::to_string(v)); }
  static QString fromStdString(const std::string &s) { return QString(s); }
  QString arg(const QString &a) const { return replace_next(a.s_); }
  template <class... R>
  QString arg(const QString &a, const QString &b, const R &...rest) const {
    return replace_next(a.s_).arg(b, rest...);
  }
  QString arg(int a) const { return replace_next(std::to_string(a)); }
  QString arg(double a) const { return replace_next(number(a).s_); }
  QString arg(double a, int width, char fmt, int prec) const { return replace_next(pad(number(a, fmt, prec).s_, width, ' ')); }
  QString arg(double a, int width, char fmt, int prec, const class QChar &fill) const;
  static int compare(const QString &a, const QString &b, int = 1) { return a.s_.compare(b.s_); }
  QString arg(int a, int width, int base, const class QChar &fill) const;
  static std::string pad(const std::string &v, int width, char fill) {
    const int n = width < 0 ? -width : width;
    if (int(v.size()) >= n) return v;
    return width < 0 ? v + std::string(n - v.size(), fill) : std::string(n - v.size(), fill) + v;
  }
  static QString number(double v, char fmt, int prec = 6) {
    char buf[64];
    char f[8] = {'%', '.', '*', fmt, 0};
    std::snprintf(buf, sizeof(buf), f, prec, v);
    return QString(buf);
  }
  std::string toStdString() const { return s_; }
  QString left(int n) const { return QString(s_.substr(0, std::max(0, n))); }
  QString right(int n) const { return QString(n >= int(s_.size()) ? s_ : s_.substr(s_.size() - n)); }
  QString mid(int p, int n = -1) const {
    if (p >= int(s_.size())) return QString();
    return QString(n < 0 ? s_.substr(p) : s_.substr(p, n));
  }
  bool startsWith(const QString &o) const { return s_.compare(0, o.s_.size(), o.s_) == 0; }
  bool endsWith(const QString &o) const {
    return s_.size() >= o.s_.size() && s_.compare(s_.size() - o.s_.size(), o.s_.size(), o.s_) == 0;
  }
  bool contains(const QString &o) const { return s_.find(o.s_) != std::string::npos; }
  int indexOf(const QString &o, int from = 0) const {
    const size_t p = s_.find(o.s_, from);
    return p == std::string::npos ? -1 : int(p);
  }
  int lastIndexOf(const QString &o) const {
    const size_t p = s_.rfind(o.s_);
    return p == std::string::npos ? -1 : int(p);
  }
  int toInt(bool *ok = nullptr, int base = 10) const {
    char *e = nullptr;
    const long v = std::strtol(s_.c_str(), &e, base);
    if (ok) *ok = e && *e == 0 && !s_.empty();
    return int(v);
  }
  double toDouble(bool *ok = nullptr) const {
    char *e = nullptr;
    const double v = std::strtod(s_.c_str(), &e);
    if (ok) *ok = e && *e == 0 && !s_.empty();
    return v;
  }
  float toFloat(bool *ok = nullptr) const { return float(toDouble(ok)); }
  void clear() { s_.clear(); }
  QString toLower() const {
    std::string r = s_;
    for (auto &c : r) c = char(std::tolower((unsigned char)c));
    return QString(r);
  }
  QString trimmed() const {
    size_t a = s_.find_first_not_of(" \t\r\n"), b = s_.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? QString() : QString(s_.substr(a, b - a + 1));
  }
  QString &replace(const QString &a, const QString &b) {
    if (a.s_.empty()) return *this;
    size_t p = 0;
    while ((p = s_.find(a.s_, p)) != std::string::npos) {
      s_.replace(p, a.s_.size(), b.s_);
      p += b.s_.size();
    }
    return *this;
  }
  QList<QString> split(const QString &sep, int = 0) const;
  const char *toLocal8Bit() const { return s_.c_str(); }
  const char *toUtf8() const { return s_.c_str(); }
  const char *toLatin1() const { return s_.c_str(); }
  bool isEmpty() const { return s_.empty(); }
  int length() const { return int(s_.size()); }
  int size() const { return int(s_.size()); }
  bool operator==(const QString &o) const { return s_ == o.s_; }
  bool operator!=(const QString &o) const { return s_ != o.s_; }
  bool operator<(const QString &o) const { return s_ < o.s_; }
  QString &operator+=(const QString &o) {
    s_ += o.s_;
    return *this;
  }
  friend QString operator+(const QString &a, const QString &b) { return QString(a.s_ + b.s_); }
  friend QString operator+(const QString &a, const char *b) { return QString(a.s_ + b); }
  friend QString operator+(const char *a, const QString &b) { return QString(a + b.s_); }

 private:
  QString replace_next(const std::string &v) const {
    for (int k = 1; k < 100; k++) {
      const std::string key = "%" + std::to_string(k);
      const size_t p = s_.find(key);
      if (p != std::string::npos) {
        std::string r = s_;
        r.replace(p, key.size(), v);
        return QString(r);
      }
    }
    return *this;
  }
  std::string s_;
};

namespace std {
template <>
struct hash<QString> {
  size_t operator()(const QString &s) const { return std::hash<std::string>()(s.toStdString()); }
};
}  // namespace std

template <class T>
class QList : public std::vector<T> {
 public:
  using std::vector<T>::vector;
  void append(const T &v) { this->push_back(v); }
  const T &at(int i) const { return (*this)[i]; }
  int size() const { return int(std::vector<T>::size()); }
  int count() const { return size(); }
  bool isEmpty() const { return this->empty(); }
  bool contains(const T &v) const { return std::find(this->begin(), this->end(), v) != this->end(); }
  int indexOf(const T &v) const {
    auto it = std::find(this->begin(), this->end(), v);
    return it == this->end() ? -1 : int(it - this->begin());
  }
  QList &operator<<(const T &v) {
    this->push_back(v);
    return *this;
  }
  const T &first() const { return this->front(); }
  const T &last() const { return this->back(); }
  void removeLast() { this->pop_back(); }
  void removeAt(int i) { this->erase(this->begin() + i); }
  void insert(int i, const T &v) { std::vector<T>::insert(this->begin() + i, v); }
  QString join(const QString &sep) const;
};
template <class T>
using QVector = QList<T>;
typedef QList<QString> QStringList;

template <class K, class V>
class QMap {
  typedef std::map<K, V> M;
  M m_;

 public:
  class iterator {
   public:
    typename M::iterator it;
    iterator() {}
    iterator(typename M::iterator i) : it(i) {}
    const K &key() const { return it->first; }
    V &value() const { return it->second; }
    V &operator*() const { return it->second; }
    V *operator->() const { return &it->second; }
    iterator &operator++() { ++it; return *this; }
    bool operator==(const iterator &o) const { return it == o.it; }
    bool operator!=(const iterator &o) const { return it != o.it; }
  };
  class const_iterator {
   public:
    typename M::const_iterator it;
    const_iterator() {}
    const_iterator(typename M::const_iterator i) : it(i) {}
    const_iterator(iterator i) : it(i.it) {}
    const K &key() const { return it->first; }
    const V &value() const { return it->second; }
    const V &operator*() const { return it->second; }
    const V *operator->() const { return &it->second; }
    const_iterator &operator++() { ++it; return *this; }
    bool operator==(const const_iterator &o) const { return it == o.it; }
    bool operator!=(const const_iterator &o) const { return it != o.it; }
  };
  iterator begin() { return iterator(m_.begin()); }
  iterator end() { return iterator(m_.end()); }
  const_iterator begin() const { return const_iterator(m_.begin()); }
  const_iterator end() const { return const_iterator(m_.end()); }
  const_iterator constBegin() const { return const_iterator(m_.begin()); }
  const_iterator constEnd() const { return const_iterator(m_.end()); }
  iterator find(const K &k) { return iterator(m_.find(k)); }
  const_iterator find(const K &k) const { return const_iterator(m_.find(k)); }
  const_iterator constFind(const K &k) const { return const_iterator(m_.find(k)); }
  iterator insert(const K &k, const V &v) {
    m_[k] = v;
    return iterator(m_.find(k));
  }
  V &operator[](const K &k) { return m_[k]; }
  V operator[](const K &k) const { return value(k); }
  bool contains(const K &k) const { return m_.find(k) != m_.end(); }
  V value(const K &k, const V &d = V()) const {
    auto it = m_.find(k);
    return it == m_.end() ? d : it->second;
  }
  int size() const { return int(m_.size()); }
  int count() const { return int(m_.size()); }
  bool isEmpty() const { return m_.empty(); }
  int remove(const K &k) { return int(m_.erase(k)); }
  void clear() { m_.clear(); }
  iterator erase(iterator i) { return iterator(m_.erase(i.it)); }
  QList<K> keys() const {
    QList<K> r;
    for (auto &kv : m_) r.push_back(kv.first);
    return r;
  }
  QList<V> values() const {
    QList<V> r;
    for (auto &kv : m_) r.push_back(kv.second);
    return r;
  }
};

template <class K, class V>
class QHash : public QMap<K, V> {};

template <class K, class V>
class QCache {
 public:
  bool insert(const K &, V *v, int = 1) {
    delete v;
    return false;
  }
  V *object(const K &) const { return nullptr; }
  bool contains(const K &) const { return false; }
};

class QDir {
 public:
  static QString separator() { return QString("/"); }
  static QString toNativeSeparators(const QString &s) { return s; }
  static QString homePath() { return QString("."); }
  static QString currentPath() { return QString("."); }
};

class QImage {
 public:
  enum Format { Format_Invalid, Format_RGB888, Format_ARGB32, Format_RGB32, Format_Grayscale8 };
  QImage() {}
  template <class... A>
  QImage(const A &...) {}
  int width() const { return 0; }
  int height() const { return 0; }
};
class QPainter {
 public:
  enum RenderHint { Antialiasing, SmoothPixmapTransform };
  QPainter(...) {}
  template <class... A>
  void drawImage(const A &...) {}
  template <class... A>
  void setRenderHint(const A &...) {}
  template <class... A>
  void setRenderHints(const A &...) {}
  void end() {}
};

class QByteArray : public std::string {
 public:
  using std::string::string;
};

namespace Qt {
enum CaseSensitivity { CaseInsensitive, CaseSensitive };
}
class QChar {
 public:
  QChar(char c = ' ') : c_(c) {}
  char c_;
  operator char() const { return c_; }
};
inline QString::QString(const QChar &c) : s_(1, c.c_) {}
inline QString QString::arg(int a, int width, int base, const QChar &fill) const {
  char buf[64];
  std::snprintf(buf, sizeof(buf), base == 16 ? "%x" : (base == 8 ? "%o" : "%d"), a);
  return replace_next(pad(buf, width, fill.c_));
}
inline QString QString::arg(double a, int width, char fmt, int prec, const QChar &fill) const {
  return replace_next(pad(number(a, fmt, prec).s_, width, fill.c_));
}
inline int qstring_compare(const QString &a, const QString &b) {
  return a.toStdString().compare(b.toStdString());
}

class QObject {
 public:
  QObject(QObject * = nullptr) {}
  virtual ~QObject() {}
  static QString tr(const char *s) { return QString(s); }
};
#define Q_OBJECT
#define signals public
#define slots
#define emit

class QMutex {
 public:
  void lock() {}
  void unlock() {}
};
class QMutexLocker {
 public:
  explicit QMutexLocker(QMutex *) {}
};

class QApplication {
 public:
  static void processEvents() {}
};

struct QLogStream {
  template <class T>
  QLogStream &operator<<(const T &) { return *this; }
  QLogStream &noquote() { return *this; }
  QLogStream &nospace() { return *this; }
};
inline QLogStream qCritical() { return QLogStream(); }
inline QLogStream qWarning() { return QLogStream(); }
inline QLogStream qDebug() { return QLogStream(); }
inline QLogStream qInfo() { return QLogStream(); }

#define Q_DECLARE_METATYPE(T)

inline QList<QString> QString::split(const QString &sep, int) const {
  QList<QString> r;
  if (sep.s_.empty()) {
    r.push_back(*this);
    return r;
  }
  size_t a = 0, p;
  while ((p = s_.find(sep.s_, a)) != std::string::npos) {
    r.push_back(QString(s_.substr(a, p - a)));
    a = p + sep.s_.size();
  }
  r.push_back(QString(s_.substr(a)));
  return r;
}
template <>
inline QString QList<QString>::join(const QString &sep) const {
  QString r;
  for (int i = 0; i < size(); i++) {
    if (i) r += sep;
    r += (*this)[i];
  }
  return r;
}
template <class A, class B>
using QPair = std::pair<A, B>;
template <class A, class B>
inline std::pair<A, B> qMakePair(const A &a, const B &b) { return std::make_pair(a, b); }
template <class T>
class QStack : public QList<T> {
 public:
  void push(const T &v) { this->push_back(v); }
  T pop() {
    T v = this->back();
    this->pop_back();
    return v;
  }
  T &top() { return this->back(); }
};
template <class T>
class QSet : public std::set<T> {
 public:
  void insert(const T &v) { std::set<T>::insert(v); }
  bool contains(const T &v) const { return this->find(v) != this->end(); }
};
class QLocale {
 public:
  QLocale() {}
  QLocale(int) {}
  enum { C = 0 };
  static QLocale system() { return QLocale(); }
  QString decimalPoint() const { return QString("."); }
  double toDouble(const QString &s, bool *ok = nullptr) const { return s.toDouble(ok); }
};
class QVariant {
 public:
  QVariant() {}
  template <class T>
  QVariant(const T &) {}
};
class QElapsedTimer {
 public:
  void start() {}
  qint64 elapsed() const { return 0; }
  qint64 nsecsElapsed() const { return 0; }
};
class QTimer : public QObject {};
class QThread : public QObject {
 public:
  enum Priority { IdlePriority, LowestPriority, LowPriority, NormalPriority, HighPriority };
  static int idealThreadCount() { return 1; }
};
class QTcpSocket : public QObject {};
class QTcpServer : public QObject {};
class QComboBox : public QObject {
 public:
  template <class... A>
  void addItem(const A &...) {}
  void clear() {}
};
enum QtMsgType { QtDebugMsg, QtWarningMsg, QtCriticalMsg, QtFatalMsg, QtInfoMsg };
class QMessageLogContext {};
#define Q_UNUSED(x) (void)(x)
inline QString tr(const char *s) { return QString(s); }

class QRect {
 public:
  QRect(int x = 0, int y = 0, int w = 0, int h = 0) : x_(x), y_(y), w_(w), h_(h) {}
  int x() const { return x_; }
  int y() const { return y_; }
  int width() const { return w_; }
  int height() const { return h_; }
  int left() const { return x_; }
  int top() const { return y_; }
  int right() const { return x_ + w_ - 1; }
  int bottom() const { return y_ + h_ - 1; }
  int x_, y_, w_, h_;
};
class QWidget : public QObject {
 public:
  double devicePixelRatioF() const { return 1.0; }
  void update() {}
  void update(const QRect &) {}
  void repaint() {}
  int width() const { return 0; }
  int height() const { return 0; }
};

// qFuzzyCompare / qFuzzyIsNull for doubles, as Qt documents them: equal when
// the difference is within 1e-12 of the smaller magnitude; null within 1e-12
inline bool qFuzzyCompare(double p1, double p2) {
  return qAbs(p1 - p2) * 1000000000000. <= qMin(qAbs(p1), qAbs(p2));
}
inline bool qFuzzyIsNull(double d) { return qAbs(d) <= 0.000000000001; }
