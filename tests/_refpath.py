# SPDX-License-Identifier: GPL-3.0-or-later
"""Puts oracle/ on sys.path (its modules are test infrastructure)."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
