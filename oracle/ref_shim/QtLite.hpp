// Qt-lite prelude (TEST INFRASTRUCTURE): the macros the reference's item headers use, reduced to
// nothing (no moc: the glue does not use Qt's meta-object system), and Qt's foreach as a range-for.
#pragma once
#include <climits>
#include <cstdint>
#include "QtGlobal"
#include "QStringList"
typedef long long qint64;
typedef unsigned long long quint64;
#define Q_OBJECT
#define Q_CLASSINFO(name, value)
#define Q_INVOKABLE
#define Q_ENUMS(x)
#ifndef foreach
#define foreach(decl, container) for (decl : container)
#endif
