"""Learned schedule cost model: data collection (collect.py), features
(features.py) and training (train.py)."""
