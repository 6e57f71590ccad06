"""Inert stand-in for matplotlib.pyplot; see matplotlib/__init__.py in this folder."""
